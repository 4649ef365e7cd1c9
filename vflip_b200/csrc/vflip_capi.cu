// C ABI of libvflip_gpu.so (declared in include/vflip.h): context, device
// buffer cache, multigrid hierarchy, V-cycle and PCG orchestration, and the
// projection / advection / transfer entry points.
//
// The PCG loop follows ivock::AMGPCGSolve (Smoke_Solver/AlgebraicMultigrid.h:
// 189-301) step for step; its scalars stay on the device and the host reads
// one small struct per iteration to test convergence.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/vflip.h"
#include "common.cuh"
#include "mg_kernels.cuh"
#include "pcg_kernels.cuh"
#include "plume_kernels.cuh"
#include "projection_kernels.cuh"
#include "transfer_kernels.cuh"
#include "smoke_kernels.cuh"
#include "learned_kernels.cuh"
#include "smoother3d.cuh"
#include "smoother_carry.cuh"
#include "coarse_direct.cuh"
#include "batch_kernels.cuh"
#include "tail_kernels.cuh"
#include "sweep_tile.cuh"
#include "tmap.h"
#include "unet_net.h"

using namespace vflip;

namespace {

constexpr int kSweepBlock = 256;
constexpr int kRedBlock = 256;
constexpr int kCoarseBlock = 1024;
constexpr int kMaxPartials = 1 << 16;
constexpr int kPcgGraphs = 4;  // PCG loop graphs kept per context
constexpr size_t kTailSmemMax = 220 * 1024;

struct Dims {
  int ni, nj, nk;
  size_t n() const { return (size_t)ni * nj * nk; }
};

// Raises a kernel's dynamic shared-memory limit on the current device, once
// per (kernel, device) pair.  The attribute is per device, so a process that
// drives several GPUs (or creates contexts from several threads) opts every
// device in; the table is guarded by a mutex.
cudaError_t smem_optin(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  const auto key = std::make_pair(func, dev);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done[key] = bytes;
  return e;
}

}  // namespace

struct vflip_ctx {
  vflip_config cfg;
  cudaStream_t stream = nullptr;
  std::string err;
  std::unordered_map<std::string, std::pair<void*, size_t>> bufs;
  bool offdiag_f32 = false;  // the operator being solved was assembled here: its couplings are FP32 values
  const void* fine_op_ready = nullptr;  // its FP32 fine-level copy, written by the assembly
  void* hbuf = nullptr;  // pinned host staging of the host-buffer entry points
  size_t hbuf_bytes = 0;
  PcgScalars* st = nullptr;         // device
  PcgScalars* st_host = nullptr;    // pinned
  double* partials = nullptr;       // device, kMaxPartials
  int* d_error = nullptr;           // device, set by kernels whose bounded waits timed out
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  int num_sms = 148;
  unsigned long long launches = 0;  // kernels launched through this context
  std::vector<vflip_ctx*> subs;     // per-system contexts of batched solves
  // the device-resident PCG loop: its graph, kept while the buffers it names stay the same
  cudaStream_t pg_stream = nullptr;
  struct PcgGraph {
    std::vector<uintptr_t> key;  // every buffer and size the captured launches name
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long init_launches = 0, body_launches = 0, tail_launches = 0;
    unsigned long long used = 0;  // last use, for replacing the least recently used
  };
  std::vector<PcgGraph> pgs;  // at most kPcgGraphs (a plain and a warm-started loop, their precisions)
  unsigned long long pg_clock = 0;
  std::unordered_map<std::string, CUtensorMap> tmaps;  // encoded TMA tensor maps by (address, shape)
  // fine-level sweep timing (vflip_set_profiling)
  bool profiling = false;
  size_t prof_fine_n = 0;
  struct ProfEvent {
    cudaEvent_t a, b;
    int tag;
  };
  std::vector<ProfEvent> prof_events;
  size_t prof_used = 0;

  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  // Cached device buffer of at least `bytes`, keyed by name.
  void* buf(const std::string& name, size_t bytes) {
    if (bytes == 0) bytes = 16;
    auto it = bufs.find(name);
    if (it != bufs.end() && it->second.second >= bytes) return it->second.first;
    if (it != bufs.end()) {
      // a buffer that has to grow gets 1/8 of headroom (rounded to 2 MiB),
      // so sizes that creep up call after call (a particle count that
      // reseeding raises a little every step) do not pay a synchronising
      // cudaFree + cudaMalloc each time
      bytes += bytes / 8;
      bytes = (bytes + (2u << 20) - 1) / (2u << 20) * (2u << 20);
      cudaFree(it->second.first);
      bufs.erase(it);
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    bufs[name] = {p, bytes};
    return p;
  }
  // Cached pinned host buffer of at least `bytes`.
  void* host_buf(size_t bytes) {
    if (hbuf && hbuf_bytes >= bytes) return hbuf;
    if (hbuf) {
      cudaStreamSynchronize(stream);
      cudaFreeHost(hbuf);
      hbuf = nullptr;
      hbuf_bytes = 0;
    }
    if (cudaMallocHost(&hbuf, bytes) != cudaSuccess) {
      hbuf = nullptr;
      return nullptr;
    }
    hbuf_bytes = bytes;
    return hbuf;
  }
};

#define VF_CUDA(call)                                                                         \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return ctx->fail(VFLIP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// Per-launch timing (vflip_set_profiling): events around the launches of
// one kind, read back by vflip_profile_kernels.  Kinds: VFLIP_PROF_*.
int prof_start(vflip_ctx* ctx, int tag, cudaStream_t stream) {
  if (!ctx->profiling) return -1;
  if (ctx->prof_used == ctx->prof_events.size()) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return -1;
    if (cudaEventCreate(&e1) != cudaSuccess) {
      cudaEventDestroy(e0);
      return -1;
    }
    ctx->prof_events.push_back({e0, e1, tag});
  }
  vflip_ctx::ProfEvent& pe = ctx->prof_events[ctx->prof_used];
  pe.tag = tag;
  if (cudaEventRecord(pe.a, stream) != cudaSuccess) return -1;
  return (int)ctx->prof_used++;
}

void prof_stop(vflip_ctx* ctx, int slot, cudaStream_t stream) {
  if (slot >= 0) cudaEventRecord(ctx->prof_events[slot].b, stream);
}

#define VF_LAUNCH_CHECK()                                                                      \
  do {                                                                                        \
    ++ctx->launches;                                                                          \
    cudaError_t e_ = cudaGetLastError();                                                      \
    if (e_ != cudaSuccess) return ctx->fail(VFLIP_ERR_CUDA, "launch: %s", cudaGetErrorString(e_)); \
  } while (0)

#define VF_ALLOC(ptr, type, name, count)                                                     \
  do {                                                                                        \
    ptr = (type*)ctx->buf((name), sizeof(type) * (size_t)(count));                           \
    if (!ptr) return ctx->fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for %s", std::string(name).c_str()); \
  } while (0)

namespace {

// f(r) over rows [0, n) on up to 32 host threads, in contiguous
// row ranges; returns the smallest row for which f returned false, or
// UINT32_MAX.  f must only write state of its own row.
template <class F>
uint32_t csr_rows_parallel(uint32_t n, F f) {
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  unsigned nt = (unsigned)std::min<uint64_t>({(uint64_t)hw, 32ull, (uint64_t)n / 65536 + 1});
  std::vector<uint32_t> first(nt, UINT32_MAX);
  auto run = [&](unsigned t) {
    uint32_t r0 = (uint32_t)((uint64_t)n * t / nt), r1 = (uint32_t)((uint64_t)n * (t + 1) / nt);
    for (uint32_t r = r0; r < r1; ++r)
      if (!f(r)) {
        first[t] = r;
        return;
      }
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < nt; ++t) pool.emplace_back(run, t);
  run(0);
  for (auto& th : pool) th.join();
  return *std::min_element(first.begin(), first.end());
}

// 1/h when h is a power of two (x*(1/h) then equals x/h exactly), else 0
double inv_pow2(double h) {
  int e;
  double m = std::frexp(h, &e);
  return (m == 0.5 && h > 0) ? 1.0 / h : 0.0;
}

int grid_for(size_t n, int block, int num_sms) {
  size_t g = (n + block - 1) / block;
  size_t cap = (size_t)num_sms * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Level sizes: ceil(n/2) per axis while the level has more than
// `max_unknowns` unknowns (GeometricLevelGen.h:44-58).
std::vector<Dims> level_dims(int ni, int nj, int nk, int max_unknowns) {
  std::vector<Dims> d{{ni, nj, nk}};
  unsigned unknowns = (unsigned)ni * nj * nk;
  while (unknowns > (unsigned)max_unknowns) {
    Dims c{(d.back().ni + 1) / 2, (d.back().nj + 1) / 2, (d.back().nk + 1) / 2};
    d.push_back(c);
    unknowns = (unsigned)c.ni * c.nj * c.nk;
  }
  return d;
}

// Typed view of one level: operator (S) and vectors (V).
template <typename S, typename V>
struct Level {
  Dims d;
  const S* diag;
  const S* xp;
  const S* yp;
  const S* zp;
  V* b;   // coarse levels own their rhs; level 0 reads the PCG residual
  V* xa;
  V* xb;
};

struct SweepShape {
  int tyo, kz, plane_stride, grid_y, grid_z;
  size_t smem;
};

template <typename A>
SweepShape sweep_shape(const Dims& d, int num_sms) {
  const int target = sizeof(A) == 8 ? 1536 : 3072;  // staged cells per plane
  int tyo = std::max(1, target / std::max(1, d.ni) - 4);
  tyo = std::min(tyo, d.nj);
  int gy = (d.nj + tyo - 1) / tyo;
  int want = num_sms * 4;
  int nz_chunks = std::max(1, std::min(d.nk, (want + gy - 1) / gy));
  int kz = std::max(4, (d.nk + nz_chunks - 1) / nz_chunks);
  kz = std::min(kz, d.nk);
  int gz = (d.nk + kz - 1) / kz;
  int rows = std::min(tyo + 4, d.nj);
  int pls = rows * d.ni;
  pls = (pls + 3) & ~3;
  SweepShape s{tyo, kz, pls, gy, gz, (size_t)4 * pls * sizeof(A)};
  return s;
}

template <typename S, typename V, bool Z, bool P, bool D>
int launch_sweep_t(vflip_ctx* ctx, const SweepArgs<S, V>& a, const SweepShape& sh) {
  auto kern = rbgs_sweep_kernel<S, V, Z, P, D, kSweepBlock>;
  if (smem_optin((const void*)kern, 200 * 1024) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the sweep's shared memory limit");
  dim3 grid(sh.grid_y, sh.grid_z);
  const int slot =
      (size_t)a.ni * a.nj * a.nk == ctx->prof_fine_n ? prof_start(ctx, VFLIP_PROF_FINE_SWEEP, ctx->stream) : -1;
  kern<<<grid, kSweepBlock, sh.smem, ctx->stream>>>(a);
  VF_LAUNCH_CHECK();
  prof_stop(ctx, slot, ctx->stream);
  return VFLIP_OK;
}

// Shape of the pipelined sweep (rbgs_sweep2_kernel): rows per tile from a
// shared-memory budget, persistent CTAs over equal shares of the level's
// (row tile, plane) pairs.
struct TmaShape {
  int tyo, gy, zlen, gz, depth, crows_max, bx, by, threads, l2_ahead, cps;
  bool carry;  // register-carry kernel (rbgs_sweep_carry_kernel)
  size_t smem;
};

constexpr size_t kTmaSmemMax = 227 * 1024 - 1024;  // opt-in limit minus the static part
// CTA sizes of the TMA-pipelined sweep: 64 x 8 or 64 x 9 threads at 256
// cells per row.  A relaxation pass walks its rows `by` at a time, so 576
// threads take the red pass of a 7-row tile (9 rows with the ring) in one
// round instead of two.
constexpr int kTmaBlock = 512, kTmaBlockWide = 576;
constexpr int kCarryNarrow = 256;  // the carry kernel on rows of <= 128 cells: 32 quads x (6 tile + 2 ring) rows

// Tile shape of the TMA-pipelined sweep.  Rows per tile, plane ranges and
// copy depth are chosen so that every CTA of a launch is resident at once
// (ctas_per_sm per SM) and marches in step with the CTAs of the neighbouring
// row tiles (their halo rows then come from L2); the 4 redundant halo planes
// of each plane range are traded against load balance.  Fields of the
// context configuration override the choice (0 = automatic).
template <typename S>
bool tma_shape(const vflip_config& cfg, const Dims& d, const Dims* cd, bool prolong, int num_sms, TmaShape& o,
               bool carry = false) {
  if (d.ni % 4 != 0 || (d.ni * sizeof(S)) % 16 != 0) return false;
  if (prolong && (!cd || cd->ni % 4 != 0)) return false;
  const int Q = (d.ni + 3) / 4;  // quads of four cells per row (one thread each)
  int bx = 1;
  while (bx < Q && bx < 128) bx <<= 1;
  // the register-carry kernel gives every (row, quad) of the red pass its own
  // thread: all quads of a row in x, the tile and its two ring rows in y
  const int cni = prolong ? cd->ni : 0;
  // one copy group in flight measured fastest at 256^3 (vflip_b200/tune.py): deeper
  // prefetch only shortens the tiles
  const int depth = cfg.smoother_depth > 0 ? std::min(cfg.smoother_depth, kTmaMaxDepth) : 1;
  auto bytes = [&](int t) { return tma_layout<S>(d.ni, t, depth, prolong ? (t + 7) / 2 : 0, cni).bytes; };
  // rows of at most 128 cells (levels that live in L2, where a CTA's march of
  // plane steps is latency-bound): the carry kernel as two 256-thread CTAs
  // per SM with 6-row tiles, so twice the CTAs each march half the planes
  const bool narrow = carry && bx == 32 && Q <= 32 && cfg.smoother_tile_rows == 0 &&
                      cfg.smoother_ctas_per_sm == 0 && bytes(kCarryNarrow / 32 - 2) <= kTmaSmemMax / 2 - 1024;
  const int carry_threads = narrow ? kCarryNarrow : kTmaBlockWide;
  if (carry && (bx < Q || carry_threads % bx != 0 || carry_threads / bx < 3)) return false;
  const int cps = narrow ? 2 : carry ? 1 : (cfg.smoother_ctas_per_sm > 0 ? std::min(cfg.smoother_ctas_per_sm, 2) : 1);
  const size_t budget = cps == 1 ? kTmaSmemMax : kTmaSmemMax / 2 - 1024;
  int tyo_max = 0;
  for (int t = 1; t <= d.nj; ++t) {
    if (bytes(t) > budget) break;
    tyo_max = t;
  }
  if (carry) tyo_max = std::min(tyo_max, carry_threads / bx - 2);
  if (tyo_max < 1) return false;
  const int slots = num_sms * cps;
  double best = 1e30;
  for (int nzr = 1; nzr <= std::min(d.nk, 16); ++nzr) {
    int gy_target = std::max(1, slots / nzr);
    int tyo = std::max((d.nj + gy_target - 1) / gy_target, 1);
    if (tyo > tyo_max) tyo = tyo_max;
    if (cfg.smoother_tile_rows > 0) tyo = std::min(cfg.smoother_tile_rows, tyo_max);
    if (cfg.smoother_plane_ranges > 0 && nzr != std::min(cfg.smoother_plane_ranges, d.nk)) continue;
    int gy = (d.nj + tyo - 1) / tyo;
    int zlen = (d.nk + nzr - 1) / nzr;
    int gz = (d.nk + zlen - 1) / zlen;
    double waves = std::ceil((double)gy * gz / slots);
    double util = (double)gy * gz / (waves * slots);
    double cost = (1.0 + 4.0 / zlen) * (1.0 + 4.0 / tyo * 0.15) / util;
    if (cost < best) {
      best = cost;
      o.tyo = tyo;
      o.gy = gy;
      o.zlen = zlen;
      o.gz = gz;
    }
  }
  if (best >= 1e30) return false;
  o.depth = depth;
  o.crows_max = prolong ? (o.tyo + 7) / 2 : 0;
  o.smem = bytes(o.tyo);
  o.bx = bx;
  o.carry = carry;
  // 576 threads take a 7-row tile's red pass in one round instead of two but
  // measured no faster at 256^3 (the copies bound the step), so 512 unless asked
  o.threads = carry ? carry_threads
                    : (cfg.smoother_threads == kTmaBlockWide && kTmaBlockWide % bx == 0 ? kTmaBlockWide : kTmaBlock);
  o.cps = cps;
  o.by = o.threads / bx;
  o.l2_ahead = cfg.smoother_prefetch < 0 ? 0 : (cfg.smoother_prefetch > 0 ? std::min(cfg.smoother_prefetch, 8) : 2);
  return o.smem <= budget;
}

template <typename S, bool Z, bool P, bool D>
int launch_tma_t(vflip_ctx* ctx, const TmaSweepArgs<S>& a, const TmaShape& sh) {
  const bool wide = sh.threads == kTmaBlockWide;
  // the tuned shape of a 256-cell-row fine level (7-row tiles, one copy group
  // in flight) runs an instance with that layout compiled in
  const bool fixed = sh.carry && a.ni == 256 && a.tyo == 7 && a.depth == 1;
  auto kern = fixed ? rbgs_sweep_carry_kernel<S, Z, P, D, kTmaBlockWide, 256, 7, 1>
                    : (sh.carry && sh.threads == kCarryNarrow) ? rbgs_sweep_carry_kernel<S, Z, P, D, kCarryNarrow>
                    : sh.carry ? rbgs_sweep_carry_kernel<S, Z, P, D, kTmaBlockWide>
                               : (wide ? rbgs_sweep_tma_kernel<S, Z, P, D, kTmaBlockWide>
                                       : rbgs_sweep_tma_kernel<S, Z, P, D, kTmaBlock>);
  if (smem_optin((const void*)kern, (int)kTmaSmemMax) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the sweep's shared memory limit");
  const int slot =
      (size_t)a.ni * a.nj * a.nk == ctx->prof_fine_n ? prof_start(ctx, VFLIP_PROF_FINE_SWEEP, ctx->stream) : -1;
  kern<<<dim3(sh.gy, sh.gz), dim3(sh.bx, sh.by), sh.smem, ctx->stream>>>(a);
  VF_LAUNCH_CHECK();
  prof_stop(ctx, slot, ctx->stream);
  return VFLIP_OK;
}

// FP32 sweeps take the TMA-pipelined kernel when the row layout allows.
template <typename S, typename V>
int sweep_tma(vflip_ctx* ctx, const Level<S, V>& L, const V* b, const V* x_in, V* x_out, const V* xc,
              const Dims* cd, double* dot_partial, int* nblocks_out, bool* used) {
  *used = false;
  if (!std::is_same<V, float>::value || std::is_same<S, double>::value || ctx->cfg.sweep_kernel == 1)
    return VFLIP_OK;
  TmaShape sh;
  const bool pro = xc != nullptr;
  // automatic (0) and 3: the register-carry kernel where its thread shape
  // fits the level, else the plain TMA kernel; 4: always the plain TMA kernel
  const bool carry = ctx->cfg.sweep_kernel == 0 || ctx->cfg.sweep_kernel == 3;
  if (!(carry && tma_shape<S>(ctx->cfg, L.d, cd, pro, ctx->num_sms, sh, true)) &&
      !tma_shape<S>(ctx->cfg, L.d, cd, pro, ctx->num_sms, sh))
    return VFLIP_OK;
  TmaSweepArgs<S> a;
  a.x_in = (const float*)x_in;
  a.x_out = (float*)x_out;
  a.b = (const float*)b;
  a.diag = L.diag;
  a.xp = L.xp;
  a.yp = L.yp;
  a.zp = L.zp;
  a.xc = (const float*)xc;
  a.ni = L.d.ni;
  a.nj = L.d.nj;
  a.nk = L.d.nk;
  a.cni = cd ? cd->ni : 0;
  a.cnj = cd ? cd->nj : 0;
  a.tyo = sh.tyo;
  a.zlen = sh.zlen;
  a.depth = sh.depth;
  a.crows_max = sh.crows_max;
  a.l2_ahead = sh.l2_ahead;
  a.dot_partial = dot_partial;
  a.error = ctx->d_error;
  if (nblocks_out) *nblocks_out = sh.gy * sh.gz;
  *used = true;
  bool zero = (x_in == nullptr), dot = (dot_partial != nullptr);
  if (zero && !pro && !dot) return launch_tma_t<S, true, false, false>(ctx, a, sh);
  if (zero && !pro && dot) return launch_tma_t<S, true, false, true>(ctx, a, sh);
  if (!zero && pro && !dot) return launch_tma_t<S, false, true, false>(ctx, a, sh);
  if (!zero && pro && dot) return launch_tma_t<S, false, true, true>(ctx, a, sh);
  if (!zero && !pro && !dot) return launch_tma_t<S, false, false, false>(ctx, a, sh);
  if (!zero && !pro && dot) return launch_tma_t<S, false, false, true>(ctx, a, sh);
  return ctx->fail(VFLIP_ERR_ARG, "sweep: prolongation needs an incoming x");
}

// Cached 3-D tensor map of a dense grid array (the address and shape fully
// determine a map, so a reused address stays valid).
const CUtensorMap* grid_map(vflip_ctx* ctx, const void* p, int es, int nx, int ny, int nz, int bx, int by) {
  char key[160];
  snprintf(key, sizeof key, "%p/%d/%d/%d/%d/%d/%d", p, es, nx, ny, nz, bx, by);
  auto it = ctx->tmaps.find(key);
  if (it != ctx->tmaps.end()) return &it->second;
  if (ctx->tmaps.size() > 4096) ctx->tmaps.clear();
  CUtensorMap m;
  if (!encode_grid_map(&m, p, es, nx, ny, nz, bx, by)) return nullptr;
  return &(ctx->tmaps[key] = m);
}

template <typename S, bool Z, bool P, bool D>
int launch_t3d_t(vflip_ctx* ctx, const T3dMaps<S>& mp, const T3dArgs& a, dim3 grid, size_t smem) {
  auto kern = rbgs_sweep_t3d_kernel<S, Z, P, D, kT3dTX, kT3dTY, kT3dBlock>;
  if (smem_optin((const void*)kern, (int)kTmaSmemMax) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the sweep's shared memory limit");
  const int slot =
      (size_t)a.ni * a.nj * a.nk == ctx->prof_fine_n ? prof_start(ctx, VFLIP_PROF_FINE_SWEEP, ctx->stream) : -1;
  kern<<<grid, kT3dBlock, smem, ctx->stream>>>(mp, a);
  VF_LAUNCH_CHECK();
  prof_stop(ctx, slot, ctx->stream);
  return VFLIP_OK;
}

// 3-D-tiled sweep (sweep_kernel == 2) when the level's rows meet the TMA
// stride and alignment rules; *used says whether it ran.
template <typename S, typename V>
int sweep_t3d(vflip_ctx* ctx, const Level<S, V>& L, const V* b, const V* x_in, V* x_out, const V* xc,
              const Dims* cd, double* dot_partial, int* nblocks_out, bool* used) {
  *used = false;
  if (ctx->cfg.sweep_kernel != 2 || !std::is_same<V, float>::value || std::is_same<S, double>::value)
    return VFLIP_OK;
  const bool pro = xc != nullptr, zero = x_in == nullptr, dot = dot_partial != nullptr;
  const int ni = L.d.ni, nj = L.d.nj, nk = L.d.nk;
  if (ni % 4 || (sizeof(S) == 2 && ni % 8) || (pro && (!cd || cd->ni % 4))) return VFLIP_OK;
  if (zero && pro) return VFLIP_OK;
  const int D = ctx->cfg.smoother_depth > 0 ? std::min(ctx->cfg.smoother_depth, kT3dMaxDepth) : 2;
  const size_t smem = t3d_smem_bytes<S, kT3dTX, kT3dTY>(D, pro);
  if (smem > kTmaSmemMax) return VFLIP_OK;
  const int ntx = (ni + kT3dTX - 1) / kT3dTX, nty = (nj + kT3dTY - 1) / kT3dTY, tiles = ntx * nty;
  const int per_sm = std::max(1, std::min(4, (int)((228 * 1024) / (smem + 2048))));
  int zr = ctx->cfg.smoother_plane_ranges > 0 ? ctx->cfg.smoother_plane_ranges
                                              : std::max(1, (ctx->num_sms * per_sm) / tiles);
  zr = std::max(1, std::min(zr, nk));
  const int zlen = (nk + zr - 1) / zr;
  zr = (nk + zlen - 1) / zlen;
  if ((size_t)tiles * zr > (size_t)kMaxPartials) return VFLIP_OK;
  using G = T3dGeom<S, kT3dTX, kT3dTY>;
  T3dMaps<S> mp;
  const CUtensorMap *mx = grid_map(ctx, zero ? (const void*)b : (const void*)x_in, 4, ni, nj, nk, G::WX, G::H),
                    *mb = grid_map(ctx, b, 4, ni, nj, nk, G::WX, G::H),
                    *md = grid_map(ctx, L.diag, sizeof(S), ni, nj, nk, G::WC, G::H),
                    *mxp = grid_map(ctx, L.xp, sizeof(S), ni, nj, nk, G::WC, G::H),
                    *myp = grid_map(ctx, L.yp, sizeof(S), ni, nj, nk, G::WC, G::H),
                    *mzp = grid_map(ctx, L.zp, sizeof(S), ni, nj, nk, G::WC, G::H);
  const CUtensorMap* mxc = pro ? grid_map(ctx, xc, 4, cd->ni, cd->nj, cd->nk, G::WXC, G::HCR) : mx;
  if (!mx || !mb || !md || !mxp || !myp || !mzp || !mxc) return VFLIP_OK;
  mp.x = *mx;
  mp.b = *mb;
  mp.d = *md;
  mp.xp = *mxp;
  mp.yp = *myp;
  mp.zp = *mzp;
  mp.xc = *mxc;
  T3dArgs a;
  a.x_out = (float*)x_out;
  a.ni = ni;
  a.nj = nj;
  a.nk = nk;
  a.cni = cd ? cd->ni : 0;
  a.cnj = cd ? cd->nj : 0;
  a.ntx = ntx;
  a.zlen = zlen;
  a.depth = D;
  a.dot_partial = dot_partial;
  a.error = ctx->d_error;
  if (nblocks_out) *nblocks_out = tiles * zr;
  *used = true;
  const dim3 grid(tiles, zr);
  if (zero && !dot) return launch_t3d_t<S, true, false, false>(ctx, mp, a, grid, smem);
  if (zero && dot) return launch_t3d_t<S, true, false, true>(ctx, mp, a, grid, smem);
  if (pro && !dot) return launch_t3d_t<S, false, true, false>(ctx, mp, a, grid, smem);
  if (pro && dot) return launch_t3d_t<S, false, true, true>(ctx, mp, a, grid, smem);
  if (!dot) return launch_t3d_t<S, false, false, false>(ctx, mp, a, grid, smem);
  return launch_t3d_t<S, false, false, true>(ctx, mp, a, grid, smem);
}

template <typename S, typename V, bool Z, bool P>
int launch_tile_t(vflip_ctx* ctx, const SweepTileArgs<S, V>& a, int tiles) {
  const int slot =
      (size_t)a.ni * a.nj * a.nk == ctx->prof_fine_n ? prof_start(ctx, VFLIP_PROF_FINE_SWEEP, ctx->stream) : -1;
  rbgs_sweep_tile_kernel<S, V, Z, P><<<tiles, kTileThreads, 0, ctx->stream>>>(a);
  VF_LAUNCH_CHECK();
  prof_stop(ctx, slot, ctx->stream);
  return VFLIP_OK;
}

// The tiled sweep (sweep_tile.cuh) on FP32 levels of at most
// tile_sweep_max_cells cells; not for a sweep that also forms z.r.
template <typename S, typename V>
int sweep_tile(vflip_ctx* ctx, const Level<S, V>& L, const V* b, const V* x_in, V* x_out, const V* xc,
               const Dims* cd, double* dot_partial, bool* used) {
  *used = false;
  if constexpr (!std::is_same<V, float>::value || std::is_same<S, double>::value) {
    return VFLIP_OK;
  } else {
    const long long n = (long long)L.d.n();
    if (dot_partial || ctx->cfg.tile_sweep_max_cells < 0 || n > ctx->cfg.tile_sweep_max_cells) return VFLIP_OK;
    const bool zero = x_in == nullptr, pro = xc != nullptr;
    if (zero && pro) return VFLIP_OK;
    SweepTileArgs<S, V> a{};
    a.x_in = x_in;
    a.x_out = x_out;
    a.b = b;
    a.diag = L.diag;
    a.xp = L.xp;
    a.yp = L.yp;
    a.zp = L.zp;
    a.xc = xc;
    a.ni = L.d.ni;
    a.nj = L.d.nj;
    a.nk = L.d.nk;
    a.cni = cd ? cd->ni : 0;
    a.cnj = cd ? cd->nj : 0;
    a.ntx = (L.d.ni + kTileTX - 1) / kTileTX;
    a.nty = (L.d.nj + kTileTY - 1) / kTileTY;
    const long long tiles = (long long)a.ntx * a.nty * ((L.d.nk + kTileTZ - 1) / kTileTZ);
    if (tiles > (1ll << 30)) return VFLIP_OK;
    *used = true;
    if (zero) return launch_tile_t<S, V, true, false>(ctx, a, (int)tiles);
    if (pro) return launch_tile_t<S, V, false, true>(ctx, a, (int)tiles);
    return launch_tile_t<S, V, false, false>(ctx, a, (int)tiles);
  }
}

// One sweep x_in -> x_out on a level; x_in == nullptr means x = 0.
template <typename S, typename V>
int sweep(vflip_ctx* ctx, const Level<S, V>& L, const V* b, const V* x_in, V* x_out, const V* xc, const Dims* cd,
          double* dot_partial, int* nblocks_out = nullptr) {
  using A = typename Num<V>::Acc;
  {
    bool used = false;
    int trc = sweep_tile<S, V>(ctx, L, b, x_in, x_out, xc, cd, dot_partial, &used);
    if (trc || used) return trc;
    int rc = sweep_t3d<S, V>(ctx, L, b, x_in, x_out, xc, cd, dot_partial, nblocks_out, &used);
    if (rc || used) return rc;
    rc = sweep_tma<S, V>(ctx, L, b, x_in, x_out, xc, cd, dot_partial, nblocks_out, &used);
    if (rc || used) return rc;
  }
  SweepShape sh = sweep_shape<A>(L.d, ctx->num_sms);
  if (sh.smem > 200 * 1024) return ctx->fail(VFLIP_ERR_ARG, "grid row of %d cells too long for one CTA", L.d.ni);
  SweepArgs<S, V> a;
  a.x_in = x_in;
  a.x_out = x_out;
  a.b = b;
  a.diag = L.diag;
  a.xp = L.xp;
  a.yp = L.yp;
  a.zp = L.zp;
  a.xc = xc;
  a.ni = L.d.ni;
  a.nj = L.d.nj;
  a.nk = L.d.nk;
  a.cni = cd ? cd->ni : 0;
  a.cnj = cd ? cd->nj : 0;
  a.tyo = sh.tyo;
  a.kz = sh.kz;
  a.plane_stride = sh.plane_stride;
  a.dot_partial = dot_partial;
  if (nblocks_out) *nblocks_out = sh.grid_y * sh.grid_z;
  if (sh.grid_y * sh.grid_z > kMaxPartials) return ctx->fail(VFLIP_ERR_ARG, "grid too large");
  bool zero = (x_in == nullptr), pro = (xc != nullptr), dot = (dot_partial != nullptr);
  if (zero && !pro && !dot) return launch_sweep_t<S, V, true, false, false>(ctx, a, sh);
  if (zero && !pro && dot) return launch_sweep_t<S, V, true, false, true>(ctx, a, sh);
  if (!zero && pro && !dot) return launch_sweep_t<S, V, false, true, false>(ctx, a, sh);
  if (!zero && pro && dot) return launch_sweep_t<S, V, false, true, true>(ctx, a, sh);
  if (!zero && !pro && !dot) return launch_sweep_t<S, V, false, false, false>(ctx, a, sh);
  if (!zero && !pro && dot) return launch_sweep_t<S, V, false, false, true>(ctx, a, sh);
  return ctx->fail(VFLIP_ERR_ARG, "sweep: prolongation needs an incoming x");
}

// FP64 band-Cholesky factor of the coarsest level (coarse_direct.cuh); `on`
// when built for this hierarchy.  *ok (device) is cleared by a singular pivot.
struct CoarseDirect {
  bool on = false;
  int bw = 0;
  double* L = nullptr;
  double* rinv = nullptr;
  int* ok = nullptr;
};
constexpr int kCholMaxBw = 160, kCholBlock = 1024, kCholSolveBlock = 256;
constexpr size_t kCholStageMax = 200 * 1024;

template <typename S, typename V>
int coarsest(vflip_ctx* ctx, const Level<S, V>& L, const V* b, V* x_out, int sweeps, double* dot_out,
             const CoarseDirect* cd = nullptr) {
  using A = typename Num<V>::Acc;
  size_t n = L.d.n();
  const int* skip = nullptr;
  if (cd && cd->on) {
    auto sk = coarse_chol_solve_kernel<V, kCholSolveBlock>;
    if (smem_optin((const void*)sk, (int)kCholStageMax) != cudaSuccess)
      return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the coarsest solve's shared memory limit");
    // the factor lives in shared memory for the solve when it fits
    const size_t staged_bytes = (n + n * (cd->bw + 1) + n) * sizeof(double);
    const int staged = staged_bytes <= kCholStageMax;
    sk<<<1, kCholSolveBlock, staged ? staged_bytes : n * sizeof(double), ctx->stream>>>(
        b, x_out, (int)n, cd->bw, cd->L, cd->rinv, cd->ok, dot_out, staged);
    VF_LAUNCH_CHECK();
    skip = cd->ok;  // the sweeps below run only if the factorisation failed
  }
  size_t smem = 6 * n * sizeof(A);
  auto kern = coarsest_rbgs_kernel<S, V, kCoarseBlock>;
  if (smem_optin((const void*)kern, 220 * 1024) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the coarsest sweeps' shared memory limit");
  if (smem > 220 * 1024) return ctx->fail(VFLIP_ERR_ARG, "coarsest level of %zu unknowns exceeds 4096", n);
  kern<<<1, kCoarseBlock, smem, ctx->stream>>>(b, L.diag, L.xp, L.yp, L.zp, x_out, L.d.ni, L.d.nj, L.d.nk, sweeps,
                                               dot_out, skip);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

template <typename S, typename V, typename VC>
int restrict_to(vflip_ctx* ctx, const Level<S, V>& L, const V* x, const V* b, VC* bc, const Dims& cd) {
  dim3 blk(32, 8);
  dim3 grid((cd.ni + 31) / 32, (cd.nj + 7) / 8, cd.nk);
  if (x)
    residual_restrict_kernel<S, V, VC, false><<<grid, blk, 0, ctx->stream>>>(
        x, b, L.diag, L.xp, L.yp, L.zp, bc, L.d.ni, L.d.nj, L.d.nk, cd.ni, cd.nj, cd.nk);
  else
    residual_restrict_kernel<S, V, VC, true><<<grid, blk, 0, ctx->stream>>>(
        x, b, L.diag, L.xp, L.yp, L.zp, bc, L.d.ni, L.d.nj, L.d.nk, cd.ni, cd.nj, cd.nk);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

// ---------------------------------------------------------------- hierarchy
// Device storage of a hierarchy in FP64 (always built: the coarsening is
// exact FP64 arithmetic) plus typed copies for the FP32/mixed modes.
struct Hierarchy64 {
  std::vector<Dims> dims;
  std::vector<double*> lv;  // 4 arrays per level, contiguous: diag, xp, yp, zp
};

int build_hierarchy64(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp,
                      const double* yp, const double* zp, Hierarchy64& H) {
  H.dims = level_dims(ni, nj, nk, ctx->cfg.coarsest_max_unknowns);
  H.lv.assign(H.dims.size(), nullptr);
  for (size_t l = 1; l < H.dims.size(); ++l) {
    double* p;
    VF_ALLOC(p, double, "h64_" + std::to_string(l), 4 * H.dims[l].n());
    H.lv[l] = p;
  }
  for (size_t l = 1; l < H.dims.size(); ++l) {
    const Dims& f = H.dims[l - 1];
    const Dims& c = H.dims[l];
    const double *fd, *fx, *fy, *fz;
    if (l == 1) {
      fd = diag; fx = xp; fy = yp; fz = zp;
    } else {
      size_t fn = f.n();
      fd = H.lv[l - 1]; fx = fd + fn; fy = fx + fn; fz = fy + fn;
    }
    size_t cn = c.n();
    double* cdp = H.lv[l];
    dim3 blk(32, 8);
    dim3 grid((c.ni + 31) / 32, (c.nj + 7) / 8, c.nk);
    galerkin_coarsen_kernel<<<grid, blk, 0, ctx->stream>>>(fd, fx, fy, fz, cdp, cdp + cn, cdp + 2 * cn,
                                                           cdp + 3 * cn, f.ni, f.nj, f.nk, c.ni, c.nj, c.nk);
    VF_LAUNCH_CHECK();
  }
  return VFLIP_OK;
}

// Typed levels: level 0 uses (S0, V), coarse levels (SC, V).
template <typename S0, typename SC, typename V>
struct Typed {
  Level<S0, V> fine;
  // the fine operator in FP64 as assembled (the outer PCG's SpMV in FP64)
  const double* d64 = nullptr;
  const double* x64 = nullptr;
  const double* y64 = nullptr;
  const double* z64 = nullptr;
  std::vector<Level<SC, V>> coarse;  // coarse[l-1] = level l
  CoarseDirect direct;               // factor of the coarsest level, when used
};

// Builds the FP64 band-Cholesky factor of the hierarchy's coarsest level
// (one CTA) when the context asks for the direct solve and the band fits.
int build_coarse_direct(vflip_ctx* ctx, const Hierarchy64& H, const double* d0, const double* x0, const double* y0,
                        const double* z0, CoarseDirect& cd, const char* tag) {
  cd.on = false;
  const int mode = ctx->cfg.coarsest_solver;
  if (mode == 1 || (mode == 0 && ctx->cfg.precision == VFLIP_PREC_FP64)) return VFLIP_OK;
  const size_t l = H.dims.size() - 1;
  const Dims& d = H.dims[l];
  const int bw = d.ni * d.nj;
  const size_t n = d.n();
  if (bw > kCholMaxBw || n > 4096) return VFLIP_OK;
  const double *dg, *xp, *yp, *zp;
  if (l == 0) {
    dg = d0; xp = x0; yp = y0; zp = z0;
  } else {
    dg = H.lv[l]; xp = dg + n; yp = xp + n; zp = yp + n;
  }
  double* p;
  VF_ALLOC(p, double, std::string(tag) + "_chol", n * (bw + 1) + n + 1);
  cd.L = p;
  cd.rinv = p + n * (bw + 1);
  cd.ok = reinterpret_cast<int*>(cd.rinv + n);
  cd.bw = bw;
  auto kern = coarse_chol_kernel<kCholBlock>;
  if (smem_optin((const void*)kern, (int)((kCholMaxBw + 1) * (kCholMaxBw + 1) * sizeof(double))) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the coarsest factorisation's shared memory limit");
  // the whole band staged beside the ring where both fit the opted-in limit
  const size_t ring = (size_t)(bw + 1) * (bw + 1), band = (size_t)n * (bw + 1);
  const bool full = ring + band <= (size_t)(kCholMaxBw + 1) * (kCholMaxBw + 1);
  kern<<<1, kCholBlock, (ring + (full ? band : 0)) * sizeof(double), ctx->stream>>>(
      dg, xp, yp, zp, d.ni, d.nj, d.nk, bw, cd.L, cd.rinv, cd.ok, full ? 1 : 0);
  VF_LAUNCH_CHECK();
  cd.on = true;
  return VFLIP_OK;
}

template <typename S, typename V>
int make_level(vflip_ctx* ctx, const Hierarchy64& H, size_t l, const double* d0, const double* x0,
               const double* y0, const double* z0, Level<S, V>& L, const char* tag) {
  L.d = H.dims[l];
  size_t n = L.d.n();
  const double *d, *x, *y, *z;
  if (l == 0) {
    d = d0; x = x0; y = y0; z = z0;
  } else {
    d = H.lv[l]; x = d + n; y = x + n; z = y + n;
  }
  if (std::is_same<S, double>::value) {
    L.diag = (const S*)d; L.xp = (const S*)x; L.yp = (const S*)y; L.zp = (const S*)z;
  } else {
    S* p;
    VF_ALLOC(p, S, std::string(tag) + "_op_" + std::to_string(l), 4 * n);
    // the assembly may have written the fine level's FP32 copy already
    if (!(l == 0 && (const void*)p == ctx->fine_op_ready)) {
      convert4_kernel<S><<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(d, x, y, z, p, n);
      VF_LAUNCH_CHECK();
    }
    L.diag = p; L.xp = p + n; L.yp = p + 2 * n; L.zp = p + 3 * n;
  }
  V* v;
  VF_ALLOC(v, V, std::string(tag) + "_vec_" + std::to_string(l), 3 * n);
  L.b = v; L.xa = v + n; L.xb = v + 2 * n;
  return VFLIP_OK;
}

template <typename S0, typename SC, typename V>
int make_typed(vflip_ctx* ctx, const Hierarchy64& H, const double* d0, const double* x0, const double* y0,
               const double* z0, Typed<S0, SC, V>& T, const char* tag) {
  int rc;
  if ((rc = make_level<S0, V>(ctx, H, 0, d0, x0, y0, z0, T.fine, tag))) return rc;
  T.d64 = d0;
  T.x64 = x0;
  T.y64 = y0;
  T.z64 = z0;
  T.coarse.resize(H.dims.size() - 1);
  for (size_t l = 1; l < H.dims.size(); ++l)
    if ((rc = make_level<SC, V>(ctx, H, l, d0, x0, y0, z0, T.coarse[l - 1], tag))) return rc;
  return build_coarse_direct(ctx, H, d0, x0, y0, z0, T.direct, tag);
}

// ---------------------------------------------------------------- V-cycle
// The first level of the one-CTA tail (tail_kernels.cuh): the first coarse
// level of at most kTailMaxCells cells, when the context runs FP32 vectors
// in the V-cycle, the tail is on, that level is not the coarsest and its
// levels fit the CTA's shared memory; else -1.
template <typename S0, typename SC, typename V>
int tail_start(const vflip_ctx* ctx, const Typed<S0, SC, V>& T, size_t* smem_bytes) {
  if (!std::is_same<V, float>::value || ctx->cfg.coarse_tail != 0) return -1;
  const int nl = (int)T.coarse.size() + 1;
  for (int l = 1; l < nl - 1; ++l) {
    if (T.coarse[l - 1].d.n() > (size_t)kTailMaxCells) continue;
    if (nl - l > kTailMaxLevels) return -1;
    size_t fl = 0;
    for (int k = l; k < nl; ++k) fl += tail_level_floats((int)T.coarse[k - 1].d.n());
    const size_t bytes = ((fl + 1) & ~(size_t)1) * sizeof(float) + T.coarse[nl - 2].d.n() * sizeof(double);
    if (bytes > kTailSmemMax) return -1;
    *smem_bytes = bytes;
    return l;
  }
  return -1;
}

// Levels t .. nl-1 in one launch: b = level t's right-hand side, x its result.
template <typename S0, typename SC, typename V>
int launch_tail(vflip_ctx* ctx, const Typed<S0, SC, V>& T, int t, size_t smem, const V* b, V* x) {
  const int nl = (int)T.coarse.size() + 1;
  TailArgs<SC, V> a{};
  a.nlev = nl - t;
  for (int k = t; k < nl; ++k) {
    const Level<SC, V>& L = T.coarse[k - 1];
    a.lv[k - t] = TailLevel<SC>{L.d.ni, L.d.nj, L.d.nk, L.diag, L.xp, L.yp, L.zp};
  }
  a.b = b;
  a.x = x;
  a.pre = ctx->cfg.pre_sweeps;
  a.post = ctx->cfg.post_sweeps;
  a.coarse_sweeps = ctx->cfg.coarse_sweeps;
  a.direct = T.direct.on ? 1 : 0;
  a.bw = T.direct.bw;
  a.L = T.direct.L;
  a.rinv = T.direct.rinv;
  a.ok = T.direct.ok;
  auto kern = tail_vcycle_kernel<SC, V>;
  if (smem_optin((const void*)kern, (int)kTailSmemMax) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the V-cycle tail's shared memory limit");
  kern<<<1, kTailThreads, smem, ctx->stream>>>(a);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

// amgVCycle (AlgebraicMultigrid.h:130-176) from x = 0.  Level l >= 1 runs
// on T.coarse[l-1].  Returns the level's final x through *xout.
template <typename S0, typename SC, typename V, typename S>
int smooth_down(vflip_ctx* ctx, const Level<S, V>& L, const V* b, V** cur_out) {
  const int pre = ctx->cfg.pre_sweeps;
  V* cur = nullptr;
  for (int s = 0; s < pre; ++s) {
    V* out = (cur == L.xa) ? L.xb : L.xa;
    int rc = sweep<S, V>(ctx, L, b, cur, out, nullptr, nullptr, nullptr);
    if (rc) return rc;
    cur = out;
  }
  *cur_out = cur;  // nullptr when pre == 0 (x = 0)
  return VFLIP_OK;
}

template <typename S, typename V>
int smooth_up(vflip_ctx* ctx, const Level<S, V>& L, const V* b, V* cur, const V* xc, const Dims& cd, V* final_out,
              double* dot_partial, int* dot_blocks, V** result) {
  const int post = ctx->cfg.post_sweeps;
  int rc;
  if (cur == nullptr) {
    // pre == 0: x is zero before prolongation; materialise x = P x_c
    cur = L.xa;
    VF_CUDA(cudaMemsetAsync(cur, 0, sizeof(V) * L.d.n(), ctx->stream));
  }
  if (post == 0) {
    dim3 blk(32, 8), grid((L.d.ni + 31) / 32, (L.d.nj + 7) / 8, L.d.nk);
    prolong_add_kernel<V, V><<<grid, blk, 0, ctx->stream>>>(cur, xc, L.d.ni, L.d.nj, L.d.nk, cd.ni, cd.nj);
    VF_LAUNCH_CHECK();
    if (final_out && final_out != cur) VF_CUDA(cudaMemcpyAsync(final_out, cur, sizeof(V) * L.d.n(),
                                                              cudaMemcpyDeviceToDevice, ctx->stream));
    *result = final_out ? final_out : cur;
    if (dot_blocks) *dot_blocks = 0;
    return VFLIP_OK;
  }
  for (int s = 0; s < post; ++s) {
    bool last = (s == post - 1);
    V* out = (last && final_out) ? final_out : ((cur == L.xa) ? L.xb : L.xa);
    rc = sweep<S, V>(ctx, L, b, cur, out, s == 0 ? xc : nullptr, &cd, last ? dot_partial : nullptr,
                     last ? dot_blocks : nullptr);
    if (rc) return rc;
    cur = out;
  }
  *result = cur;
  return VFLIP_OK;
}

// z = V(r); when want_dot, rho_new = z.r is reduced into the PCG scalars.
template <typename S0, typename SC, typename V>
int vcycle(vflip_ctx* ctx, Typed<S0, SC, V>& T, const V* r, V* z, bool want_dot) {
  int rc;
  const int nl = (int)T.coarse.size() + 1;
  if (nl == 1) {
    rc = coarsest<S0, V>(ctx, T.fine, r, z, ctx->cfg.coarse_sweeps, want_dot ? ctx->partials : nullptr,
                         &T.direct);
    if (rc) return rc;
    if (want_dot) {
      fold_kernel<kRedBlock><<<1, kRedBlock, 0, ctx->stream>>>(ctx->partials, 1, ctx->st, kReduceRho, 0.0);
      VF_LAUNCH_CHECK();
    }
    return VFLIP_OK;
  }
  std::vector<V*> after_pre(nl, nullptr);
  size_t tail_smem = 0;
  const int t = tail_start(ctx, T, &tail_smem);
  const int bottom = t > 0 ? t : nl - 1;  // the levels from here down run as one unit
  const int vslot = prof_start(ctx, VFLIP_PROF_VCYCLE, ctx->stream);
  // down
  if ((rc = smooth_down<S0, SC, V, S0>(ctx, T.fine, r, &after_pre[0]))) return rc;
  if ((rc = restrict_to<S0, V, V>(ctx, T.fine, after_pre[0], r, T.coarse[0].b, T.coarse[0].d))) return rc;
  const int cslot = prof_start(ctx, VFLIP_PROF_COARSE, ctx->stream);
  for (int l = 1; l < bottom; ++l) {
    Level<SC, V>& L = T.coarse[l - 1];
    if ((rc = smooth_down<S0, SC, V, SC>(ctx, L, L.b, &after_pre[l]))) return rc;
    if ((rc = restrict_to<SC, V, V>(ctx, L, after_pre[l], L.b, T.coarse[l].b, T.coarse[l].d))) return rc;
  }
  // bottom: the coarsest level, or the one-CTA tail from level t down
  Level<SC, V>& B = T.coarse[bottom - 1];
  if (t > 0) {
    if ((rc = launch_tail(ctx, T, t, tail_smem, B.b, B.xa))) return rc;
  } else if ((rc = coarsest<SC, V>(ctx, B, B.b, B.xa, ctx->cfg.coarse_sweeps, nullptr, &T.direct))) {
    return rc;
  }
  V* xc = B.xa;
  Dims cd = B.d;
  // up
  for (int l = bottom - 1; l >= 1; --l) {
    Level<SC, V>& L = T.coarse[l - 1];
    V* res;
    if ((rc = smooth_up<SC, V>(ctx, L, L.b, after_pre[l], xc, cd, nullptr, nullptr, nullptr, &res))) return rc;
    xc = res;
    cd = L.d;
  }
  prof_stop(ctx, cslot, ctx->stream);
  int dot_blocks = 0;
  V* res;
  if ((rc = smooth_up<S0, V>(ctx, T.fine, r, after_pre[0], xc, cd, z, want_dot ? ctx->partials : nullptr,
                             &dot_blocks, &res)))
    return rc;
  prof_stop(ctx, vslot, ctx->stream);
  if (want_dot) {
    if (dot_blocks > 0) {
      fold_kernel<kRedBlock><<<1, kRedBlock, 0, ctx->stream>>>(ctx->partials, dot_blocks, ctx->st, kReduceRho, 0.0);
    } else {
      size_t n = T.fine.d.n();
      dot_kernel<V, kRedBlock><<<grid_for(n, kRedBlock, ctx->num_sms), kRedBlock, 0, ctx->stream>>>(
          z, r, n, ctx->partials, ctx->st, kReduceRho);
    }
    VF_LAUNCH_CHECK();
  }
  return VFLIP_OK;
}

// ---------------------------------------------------------------- PCG
// Device-side failure report of the pipelined smoother (a bounded wait that
// timed out); read after a synchronisation.
int check_kernel_error(vflip_ctx* ctx, int err_host) {
  if (err_host) {
    cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream);
    return ctx->fail(VFLIP_ERR_CUDA, "smoother copy pipeline timed out");
  }
  return VFLIP_OK;
}

int read_scalars(vflip_ctx* ctx) {
  VF_CUDA(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(PcgScalars), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaMemcpyAsync(&ctx->st_host->kernel_error, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  return check_kernel_error(ctx, ctx->st_host->kernel_error);
}

// s_new = z + beta s_old (s_new = z on the first iteration), q = A s_new on
// the fine level and the s.q reduction (alpha).  The plane-marching kernel
// runs where the fine rows are whole warps of quads (unless the context asks
// for the column kernel, or `plane` is false: the batched graph keeps the
// column kernel); both give the same q and s_new bits.
template <typename W, typename Z = W, typename O = W>
int launch_spmv_dot(vflip_ctx* ctx, cudaStream_t stream, bool first, const Z* z, const W* s_old, W* s_new, W* q,
                    const W* diag, const O* xp, const O* yp, const O* zp, const Dims& d, bool plane = true) {
  const int nq = d.ni / 4;
  if (plane && ctx->cfg.spmv_kernel == 0 && d.ni % 128 == 0 && nq <= 256) {
    // about 384 threads a block (at 256 cells a row: 4 rows + 2 halo rows,
    // three blocks per SM) and two waves of blocks measured fastest
    const int ty = std::max(2, 384 / nq - 2);
    const int rows = ty + 2;
    const size_t smem = 3 * (size_t)rows * nq * (sizeof(Quad<W>) + sizeof(Quad<O>));
    auto kern = first ? pcg_spmv_dot_plane_kernel<W, true, Z, O> : pcg_spmv_dot_plane_kernel<W, false, Z, O>;
    if (smem_optin((const void*)kern, (int)smem) != cudaSuccess)
      return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the SpMV kernel's shared memory limit");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nq * rows, smem) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    // row tiles x plane ranges
    const int rt = (d.nj + ty - 1) / ty;
    int kr = std::max(1, std::min(d.nk, 2 * per_sm * ctx->num_sms / rt));
    const int kz = (d.nk + kr - 1) / kr;
    kr = (d.nk + kz - 1) / kz;
    if ((size_t)rt * kr <= (size_t)kMaxPartials) {
      const int slot = prof_start(ctx, VFLIP_PROF_SPMV, stream);
      kern<<<dim3(rt, kr), dim3(nq, rows), smem, stream>>>(z, s_old, s_new, q, diag, xp, yp, zp, d.ni, d.nj, d.nk,
                                                           ty, kz, ctx->partials, ctx->st);
      prof_stop(ctx, slot, stream);
      VF_LAUNCH_CHECK();
      return VFLIP_OK;
    }
  }
  dim3 sblk(kRedBlock);
  const int kz = 8;
  dim3 sgrid((d.ni + 31) / 32, (d.nj + kRedBlock / 32 - 1) / (kRedBlock / 32), (d.nk + kz - 1) / kz);
  if ((size_t)sgrid.x * sgrid.y * sgrid.z > (size_t)kMaxPartials) return ctx->fail(VFLIP_ERR_ARG, "grid too large");
  const int slot = prof_start(ctx, VFLIP_PROF_SPMV, stream);
  if (first)
    pcg_spmv_dot_kernel<W, true, kRedBlock, Z, O><<<sgrid, sblk, 0, stream>>>(z, s_old, s_new, q, diag, xp, yp, zp,
                                                                           d.ni, d.nj, d.nk, kz, ctx->partials,
                                                                           ctx->st);
  else
    pcg_spmv_dot_kernel<W, false, kRedBlock, Z, O><<<sgrid, sblk, 0, stream>>>(z, s_old, s_new, q, diag, xp, yp, zp,
                                                                            d.ni, d.nj, d.nk, kz, ctx->partials,
                                                                            ctx->st);
  prof_stop(ctx, slot, stream);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

// The outer PCG's vectors: W = V (everything in the working precision) or
// W = double around a narrower V-cycle (FP32/MIXED contexts by default).
// In the second case x is the caller's FP64 result itself, r/s/q are FP64,
// the SpMV uses the FP64 fine operator, and rv is r rounded to V for the
// V-cycle (written by the update).
template <typename W, typename V>
struct OuterVecs {
  W *x = nullptr, *r = nullptr, *s0 = nullptr, *s1 = nullptr, *q = nullptr;
  V *rv = nullptr, *z = nullptr;
  const W *od = nullptr, *ox = nullptr, *oy = nullptr, *oz = nullptr;
  // the FP32 fine operator's couplings, read instead of ox/oy/oz when they
  // equal the FP64 ones (an operator the library assembled: every coupling
  // is a float value, so its FP32 copy is exact)
  const float *fx = nullptr, *fy = nullptr, *fz = nullptr;
};

template <typename W, typename S0, typename SC, typename V>
int outer_vecs(vflip_ctx* ctx, Typed<S0, SC, V>& T, double* result, OuterVecs<W, V>& o) {
  const size_t n = T.fine.d.n();
  constexpr bool same = std::is_same<W, V>::value;
  VF_ALLOC(o.z, V, "pcg_z", n);
  VF_ALLOC(o.s0, W, same ? "pcg_s0" : "pcg_s0_64", n);
  VF_ALLOC(o.s1, W, same ? "pcg_s1" : "pcg_s1_64", n);
  VF_ALLOC(o.q, W, same ? "pcg_q" : "pcg_q_64", n);
  if constexpr (same) {
    VF_ALLOC(o.x, W, "pcg_x", n);
    VF_ALLOC(o.r, W, "pcg_r", n);
    o.rv = o.r;
    o.od = reinterpret_cast<const W*>(T.fine.diag);
    o.ox = reinterpret_cast<const W*>(T.fine.xp);
    o.oy = reinterpret_cast<const W*>(T.fine.yp);
    o.oz = reinterpret_cast<const W*>(T.fine.zp);
  } else {
    o.x = result;
    VF_ALLOC(o.r, W, "pcg_r_64", n);
    VF_ALLOC(o.rv, V, "pcg_r", n);
    o.od = T.d64;
    o.ox = T.x64;
    o.oy = T.y64;
    o.oz = T.z64;
    if constexpr (std::is_same<S0, float>::value) {
      if (ctx->offdiag_f32) {
        o.fx = T.fine.xp;
        o.fy = T.fine.yp;
        o.fz = T.fine.zp;
      }
    }
  }
  return VFLIP_OK;
}

// The outer PCG's s = z + beta s, q = A s and s.q, on the FP32 couplings
// where they are exact (bitwise the same q).
template <typename W, typename V>
int outer_spmv(vflip_ctx* ctx, cudaStream_t stream, bool first, const OuterVecs<W, V>& o, const W* s_old, W* s_new,
               W* q, const Dims& d) {
  if constexpr (!std::is_same<W, float>::value) {
    if (o.fx) return launch_spmv_dot<W, V, float>(ctx, stream, first, o.z, s_old, s_new, q, o.od, o.fx, o.fy, o.fz, d);
  }
  return launch_spmv_dot<W, V>(ctx, stream, first, o.z, s_old, s_new, q, o.od, o.ox, o.oy, o.oz, d);
}

// r = rhs, x = 0, |rhs|_inf
template <typename W, typename V>
void launch_pcg_init(vflip_ctx* ctx, cudaStream_t st, const OuterVecs<W, V>& o, const double* rhs, size_t n,
                     double tol_factor) {
  const int gb = grid_for(n, kRedBlock, ctx->num_sms);
  if constexpr (std::is_same<W, V>::value)
    pcg_init_kernel<V, kRedBlock><<<gb, kRedBlock, 0, st>>>(rhs, o.r, o.x, n, ctx->partials, ctx->st, tol_factor);
  else
    pcg_init_outer_kernel<V, kRedBlock><<<gb, kRedBlock, 0, st>>>(rhs, o.r, o.rv, o.x, n, ctx->partials, ctx->st,
                                                                  tol_factor);
}

// x += alpha s, r -= alpha q, |r|_inf (and the V-cycle's copy of r)
template <typename W, typename V>
void launch_pcg_update(vflip_ctx* ctx, cudaStream_t st, const OuterVecs<W, V>& o, const W* s, size_t n) {
  const int gb = grid_for(n, kRedBlock, ctx->num_sms);
  if constexpr (std::is_same<W, V>::value)
    pcg_update_kernel<V, kRedBlock><<<gb, kRedBlock, 0, st>>>(o.x, o.r, s, o.q, n, ctx->partials, ctx->st);
  else
    pcg_update_outer_kernel<V, kRedBlock><<<gb, kRedBlock, 0, st>>>(o.x, o.r, o.rv, s, o.q, n, ctx->partials,
                                                                    ctx->st);
}

// AMGPCGSolve's loop on the device (AlgebraicMultigrid.h:253-286): a CUDA
// graph of [r = rhs, x = 0, |rhs|] -> while node {V-cycle with the fused z.r
// (beta), s = z + beta s, q = A s with s.q (alpha), x/r update with |r|_inf,
// stop test} -> x to FP64, captured once and relaunched while the buffers
// and the hierarchy's layout stay the same; the host reads the scalars once.
// The loop body rotates the host loop (the V-cycle first, s = 0 on entry),
// so the iterates are the host loop's.  *done is false when the solve did
// not converge (zero or NaN rho, max_iterations): the caller then repeats it
// with the host loop, whose early exits set the result as the reference's.
template <typename W, typename S0, typename SC, typename V>
int pcg_solve_graph(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol_factor,
                    int maxit, vflip_solve_stats* stats, bool* done, bool warm = false) {
  *done = false;
  const Dims d = T.fine.d;
  const size_t n = d.n();
  OuterVecs<W, V> o;
  int rc0;
  if ((rc0 = outer_vecs<W>(ctx, T, result, o))) return rc0;
  W *x = o.x, *r = o.r, *s = o.s0, *q = o.q;
  V* z = o.z;
  int* itp;
  VF_ALLOC(itp, int, "pcg_it", 1);
  // everything the captured launches name
  std::vector<uintptr_t> key;
  auto kp = [&](const void* p) { key.push_back((uintptr_t)p); };
  auto kl = [&](const auto& L) {
    kp(L.diag); kp(L.xp); kp(L.yp); kp(L.zp); kp(L.b); kp(L.xa); kp(L.xb);
    key.push_back((uintptr_t)L.d.ni); key.push_back((uintptr_t)L.d.nj); key.push_back((uintptr_t)L.d.nk);
  };
  kp(rhs); kp(result); kp(x); kp(r); kp(o.rv); kp(z); kp(s); kp(q); kp(itp); kp(ctx->st); kp(ctx->partials);
  kp(o.od); kp(o.ox); kp(o.oy); kp(o.oz); kp(o.fx); kp(o.fy); kp(o.fz);
  kl(T.fine);
  for (const auto& L : T.coarse) kl(L);
  kp(T.direct.L); kp(T.direct.rinv); kp(T.direct.ok);
  key.push_back((uintptr_t)T.direct.on); key.push_back((uintptr_t)T.direct.bw); key.push_back((uintptr_t)maxit);
  key.push_back((uintptr_t)warm);
  uint64_t tb;
  std::memcpy(&tb, &tol_factor, sizeof tb);
  key.push_back((uintptr_t)tb);
  const int gb = grid_for(n, kRedBlock, ctx->num_sms);
  vflip_ctx::PcgGraph* E = nullptr;
  for (auto& g : ctx->pgs)
    if (g.exec && g.key == key) E = &g;
  if (!E) {
    if (ctx->pgs.size() < (size_t)kPcgGraphs) {
      ctx->pgs.emplace_back();
      E = &ctx->pgs.back();
    } else {
      E = &*std::min_element(ctx->pgs.begin(), ctx->pgs.end(),
                             [](const vflip_ctx::PcgGraph& a, const vflip_ctx::PcgGraph& b) { return a.used < b.used; });
      if (E->exec) cudaGraphExecDestroy(E->exec);
      if (E->graph) cudaGraphDestroy(E->graph);
      *E = vflip_ctx::PcgGraph{};
    }
    if (!ctx->pg_stream) VF_CUDA(cudaStreamCreateWithFlags(&ctx->pg_stream, cudaStreamNonBlocking));
    const cudaStream_t cs = ctx->pg_stream;
    cudaGraph_t graph = nullptr;
    VF_CUDA(cudaGraphCreate(&graph, 0));
    E->graph = graph;
    cudaGraphConditionalHandle hnd;
    VF_CUDA(cudaGraphConditionalHandleCreate(&hnd, graph, 0, 0));
    const cudaStream_t saved = ctx->stream;
    const bool prof = ctx->profiling;
    ctx->stream = cs;
    ctx->profiling = false;
    auto restore = [&](int code) {
      ctx->stream = saved;
      ctx->profiling = prof;
      return code;
    };
    auto end_capture = [&](cudaGraph_t g) -> int {
      cudaGraph_t out = nullptr;
      const cudaError_t e = cudaStreamEndCapture(cs, &out);
      if (e != cudaSuccess || out != g)
        return ctx->fail(VFLIP_ERR_CUDA, "PCG loop capture failed: %s", cudaGetErrorString(e));
      return VFLIP_OK;
    };
    int rc;
    const unsigned long long before_capture = ctx->launches;
    if (cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return restore(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCaptureToGraph"));
    // warm: the caller has set x, r, its V copy and the scalars (tolerance
    // and |r|_inf of the initial guess); otherwise r = b, x = 0
    if (!warm) cudaMemsetAsync(ctx->st, 0, sizeof(PcgScalars), cs);
    cudaMemsetAsync(s, 0, n * sizeof(W), cs);
    if (!warm) launch_pcg_init(ctx, cs, o, rhs, n, tol_factor);
    pcg_loop_init_kernel<<<1, 32, 0, cs>>>(ctx->st, itp, hnd);
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    if (cudaStreamGetCaptureInfo(cs, &cst, nullptr, nullptr, &deps, &ndeps) != cudaSuccess) {
      end_capture(graph);
      return restore(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamGetCaptureInfo"));
    }
    std::vector<cudaGraphNode_t> dv(deps, deps + ndeps);
    if ((rc = end_capture(graph))) return restore(rc);
    E->init_launches = warm ? 1 : 2;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hnd;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    if (cudaGraphAddNode(&wn, graph, dv.data(), dv.size(), &cp) != cudaSuccess)
      return restore(ctx->fail(VFLIP_ERR_CUDA, "cannot add the while node"));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return restore(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCaptureToGraph (body)"));
    const unsigned long long l0 = ctx->launches;
    int brc = vcycle<S0, SC, V>(ctx, T, o.rv, z, true);
    if (!brc) {
      pcg_direction_kernel<W, V><<<grid_for(n, 256, ctx->num_sms), 256, 0, cs>>>(z, s, n, ctx->st);
      ++ctx->launches;
      if (o.fx)
        brc = launch_spmv_dot<W, W, float>(ctx, cs, true, (const W*)s, (const W*)nullptr, (W*)nullptr, q, o.od, o.fx,
                                           o.fy, o.fz, d);
      else
        brc = launch_spmv_dot<W>(ctx, cs, true, (const W*)s, (const W*)nullptr, (W*)nullptr, q, o.od, o.ox, o.oy,
                                 o.oz, d);
    }
    if (!brc) {
      launch_pcg_update(ctx, cs, o, s, n);
      pcg_loop_cond_kernel<<<1, 32, 0, cs>>>(ctx->st, itp, maxit, hnd);
      ctx->launches += 2;
    }
    if ((rc = end_capture(body))) return restore(rc);
    if (brc) return restore(brc);
    E->body_launches = ctx->launches - l0;
    if (cudaStreamBeginCaptureToGraph(cs, graph, &wn, nullptr, 1, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return restore(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCaptureToGraph (result)"));
    if constexpr (std::is_same<W, V>::value) {
      to_double_kernel<V, kRedBlock><<<gb, kRedBlock, 0, cs>>>(x, result, n);
      E->tail_launches = 1;
    } else {
      E->tail_launches = 0;  // x is the result
    }
    if ((rc = end_capture(graph))) return restore(rc);
    restore(VFLIP_OK);
    ctx->launches = before_capture;  // captured launches count when the graph runs
    if (cudaGraphInstantiate(&E->exec, graph, 0) != cudaSuccess) {
      E->exec = nullptr;
      return ctx->fail(VFLIP_ERR_CUDA, "cudaGraphInstantiate failed (PCG loop)");
    }
    E->key = key;
  }
  E->used = ++ctx->pg_clock;
  if (cudaGraphLaunch(E->exec, ctx->stream) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cudaGraphLaunch (PCG loop)");
  int iters = 0;
  VF_CUDA(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(PcgScalars), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaMemcpyAsync(&ctx->st_host->kernel_error, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  VF_CUDA(cudaMemcpyAsync(&iters, itp, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  int rc;
  if ((rc = check_kernel_error(ctx, ctx->st_host->kernel_error))) return rc;
  const PcgScalars& h = *ctx->st_host;
  ctx->launches += E->init_launches + (unsigned long long)iters * E->body_launches + E->tail_launches;
  const bool ok = h.converged && !h.bad_rho;
  // a failed plain solve is repeated by the host loop (its exact statistics);
  // a failed warm start is reported as such (the caller decides what follows)
  if (!ok && !warm) return VFLIP_OK;
  if (stats) {
    stats->iterations = iters;
    stats->vcycles = iters;
    stats->levels = (int)T.coarse.size() + 1;
    stats->converged = ok ? 1 : 0;
    stats->residual = h.res;
    stats->rhs_norm = h.rhs_norm;
  }
  *done = true;
  return ok ? VFLIP_OK : VFLIP_NOT_CONVERGED;
}

// AMGPCGSolve (AlgebraicMultigrid.h:189-301) with the outer vectors in W.
// warm: the caller has set x (the result), r, its V copy and the scalars
// (tolerance from |rhs|_inf, |r|_inf of the initial guess).
template <typename W, typename S0, typename SC, typename V>
int pcg_solve_w(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol_factor,
                int maxit, vflip_solve_stats* stats, V* x1_out, bool warm = false) {
  constexpr bool same = std::is_same<W, V>::value;
  if (ctx->cfg.pcg_loop == 0 && !ctx->profiling && !x1_out) {
    bool done = false;
    const int grc = pcg_solve_graph<W>(ctx, T, rhs, result, tol_factor, maxit, stats, &done, warm);
    if (grc < 0 || done) return grc;
  }
  const Dims d = T.fine.d;
  const size_t n = d.n();
  OuterVecs<W, V> o;
  int rc;
  if ((rc = outer_vecs<W>(ctx, T, result, o))) return rc;
  const int gb = grid_for(n, kRedBlock, ctx->num_sms);
  if (!warm) {
    VF_CUDA(cudaMemsetAsync(ctx->st, 0, sizeof(PcgScalars), ctx->stream));
    launch_pcg_init(ctx, ctx->stream, o, rhs, n, tol_factor);
    VF_LAUNCH_CHECK();
  }
  if ((rc = read_scalars(ctx))) return rc;
  PcgScalars& h = *ctx->st_host;
  const double rhs_norm = warm ? h.rhs_norm : h.res;
  int iterations = 0, vcycles = 0;
  double residual = h.res;
  auto finish = [&](int st_code) -> int {
    if constexpr (same) {
      to_double_kernel<V, kRedBlock><<<gb, kRedBlock, 0, ctx->stream>>>(o.x, result, n);
      ++ctx->launches;
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return ctx->fail(VFLIP_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    }
    if (stats) {
      stats->iterations = iterations;
      stats->vcycles = vcycles;
      stats->levels = (int)T.coarse.size() + 1;
      stats->converged = st_code == VFLIP_OK ? 1 : 0;
      stats->residual = residual;
      stats->rhs_norm = rhs_norm;
    }
    return st_code;
  };
  if (h.res == 0.0 || (warm && h.converged)) {  // AlgebraicMultigrid.h:214-232
    iterations = 0;
    return finish(VFLIP_OK);
  }
  if ((rc = vcycle<S0, SC, V>(ctx, T, o.rv, o.z, true))) return rc;
  ++vcycles;
  if ((rc = read_scalars(ctx))) return rc;
  if (h.bad_rho) {  // AlgebraicMultigrid.h:236-252
    iterations = 0;
    return finish(VFLIP_NOT_CONVERGED);
  }
  W* s_old = o.s0;
  W* s_new = o.s1;
  int it;
  for (it = 0; it < maxit; ++it) {
    if ((rc = outer_spmv<W, V>(ctx, ctx->stream, it == 0, o, s_old, s_new, o.q, d)))
      return rc;
    const int uslot = prof_start(ctx, VFLIP_PROF_UPDATE, ctx->stream);
    launch_pcg_update(ctx, ctx->stream, o, s_new, n);
    prof_stop(ctx, uslot, ctx->stream);
    VF_LAUNCH_CHECK();
    if (it == 0 && x1_out) {
      if constexpr (same) {
        VF_CUDA(cudaMemcpyAsync(x1_out, o.x, n * sizeof(V), cudaMemcpyDeviceToDevice, ctx->stream));
      } else {
        convert_kernel<V><<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(o.x, x1_out, n);
        VF_LAUNCH_CHECK();
      }
    }
    if ((rc = read_scalars(ctx))) return rc;
    residual = h.res;
    if (h.converged) {
      iterations = it + 1;
      return finish(VFLIP_OK);
    }
    if ((rc = vcycle<S0, SC, V>(ctx, T, o.rv, o.z, true))) return rc;
    ++vcycles;
    std::swap(s_old, s_new);
  }
  iterations = it;
  return finish(VFLIP_NOT_CONVERGED);
}

// The outer loop runs in FP64 around an FP32/MIXED V-cycle unless the
// context asks for the working precision (pcg_vectors = 1).
template <typename S0, typename SC, typename V>
int pcg_solve(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol_factor, int maxit,
              vflip_solve_stats* stats, V* x1_out = nullptr) {
  if constexpr (!std::is_same<V, double>::value) {
    if (ctx->cfg.pcg_vectors == 0) return pcg_solve_w<double>(ctx, T, rhs, result, tol_factor, maxit, stats, x1_out);
  }
  return pcg_solve_w<V>(ctx, T, rhs, result, tol_factor, maxit, stats, x1_out);
}

// ---------------------------------------------------------------- learned
// Options of a learned-preconditioned projection (vflip_project_learned).
struct LearnedOpts {
  vflip::unet::Net* net = nullptr;
  int mode = 0;
  int level = 1;
  const double* diag = nullptr;  // fine FP64 diagonal: fluid cells are diag > 0
  float* s_in2 = nullptr;        // capture outputs (network grid)
  float* s_tgt2 = nullptr;
  float* s_w = nullptr;
  vflip_learned_stats* lstats = nullptr;
};

// in2 = (s R^L rhs, R^L fluid), s = 1/|R^L rhs|_inf (device scalar); mc keeps R^L fluid
int learned_features(vflip_ctx* ctx, const LearnedOpts& lo, const Dims& d, const double* rhs, int X, int Y, int Z,
                     float* in2, float** mc_out, double** scale_out) {
  const size_t nv = (size_t)X * Y * Z;
  float *bc, *mc;
  double* scale;
  unsigned int* counter;
  VF_ALLOC(bc, float, "lrn_bc", nv);
  VF_ALLOC(mc, float, "lrn_mc", nv);
  VF_ALLOC(scale, double, "lrn_scale", 1);
  VF_ALLOC(counter, unsigned int, "lrn_counter", 1);
  const int g = grid_for(nv, 256, ctx->num_sms);
  block_average_kernel<double, double><<<g, 256, 0, ctx->stream>>>(rhs, nullptr, 0, d.ni, d.nj, d.nk, lo.level, bc,
                                                                    X, Y, Z);
  VF_LAUNCH_CHECK();
  block_average_kernel<double, double><<<g, 256, 0, ctx->stream>>>(lo.diag, nullptr, 1, d.ni, d.nj, d.nk, lo.level,
                                                                    mc, X, Y, Z);
  VF_LAUNCH_CHECK();
  VF_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), ctx->stream));
  const int gr = std::min(grid_for(nv, kRedBlock, ctx->num_sms), kMaxPartials);
  inv_absmax_kernel<kRedBlock><<<gr, kRedBlock, 0, ctx->stream>>>(bc, nv, ctx->partials, counter, scale);
  VF_LAUNCH_CHECK();
  pack2_kernel<<<g, 256, 0, ctx->stream>>>(bc, mc, scale, 0, in2, nv);
  VF_LAUNCH_CHECK();
  *mc_out = mc;
  *scale_out = scale;
  return VFLIP_OK;
}

// Training triple of a converged plain solve: features, targets
// (s R^L p, s R^L (p - x1)) and weight R^L fluid, on the network grid.
template <typename V>
int learned_capture(vflip_ctx* ctx, const LearnedOpts& lo, const Dims& d, const double* rhs, const double* p,
                    const V* x1) {
  int X, Y, Z;
  learned_grid_dims(d.ni, d.nj, d.nk, lo.level, X, Y, Z);
  const size_t nv = (size_t)X * Y * Z;
  float *mc, *pc, *dc;
  double* scale;
  int rc;
  if ((rc = learned_features(ctx, lo, d, rhs, X, Y, Z, lo.s_in2, &mc, &scale))) return rc;
  VF_ALLOC(pc, float, "lrn_pc", nv);
  VF_ALLOC(dc, float, "lrn_dc", nv);
  const int g = grid_for(nv, 256, ctx->num_sms);
  block_average_kernel<double, double><<<g, 256, 0, ctx->stream>>>(p, nullptr, 0, d.ni, d.nj, d.nk, lo.level, pc, X,
                                                                    Y, Z);
  VF_LAUNCH_CHECK();
  block_average_kernel<double, V><<<g, 256, 0, ctx->stream>>>(p, x1, 2, d.ni, d.nj, d.nk, lo.level, dc, X, Y, Z);
  VF_LAUNCH_CHECK();
  pack2_kernel<<<g, 256, 0, ctx->stream>>>(pc, dc, scale, 1, lo.s_tgt2, nv);
  VF_LAUNCH_CHECK();
  VF_CUDA(cudaMemcpyAsync(lo.s_w, mc, nv * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  return VFLIP_OK;
}

// Energy-minimising coefficients over the active subset of the Ritz
// vectors: G gamma = g with G_ij = w_i.A w_j (upper triangle first in
// `dots`, then g_i = w_i.b); vectors whose pivot collapses (linearly
// dependent, zero, or non-finite) are dropped.  Returns the kept count.
__host__ __device__ inline bool finite_d(double v) { return (v - v) == 0.0; }

// gamma = argmin of the energy over the subspace of the vectors in use:
// G gamma = W^T b by Cholesky of the diagonally scaled Gram matrix, dropping
// a vector whose pivot is not positive or not finite and starting again.
// Returns the subspace dimension (0: gamma = 0).
__host__ __device__ int ritz_solve(const double* dots, const bool* use, double* gamma) {
  constexpr int M = kRitzVecs;
  double G[M][M], g[M];
  int k = 0;
  for (int a = 0; a < M; ++a)
    for (int c = a; c < M; ++c) G[a][c] = G[c][a] = dots[k++];
  for (int a = 0; a < M; ++a) g[a] = dots[k++];
  bool on[M];
  for (int i = 0; i < M; ++i) {
    gamma[i] = 0.0;
    on[i] = use[i] && G[i][i] > 0.0 && finite_d(G[i][i]) && finite_d(g[i]);
  }
  for (int attempt = 0; attempt < M; ++attempt) {
    int idx[M], m = 0;
    for (int i = 0; i < M; ++i)
      if (on[i]) idx[m++] = i;
    if (m == 0) return 0;
    // Cholesky of the diagonally scaled subset
    double L[M][M] = {}, sc[M];
    for (int a = 0; a < m; ++a) sc[a] = 1.0 / sqrt(G[idx[a]][idx[a]]);
    int bad = -1;
    for (int a = 0; a < m && bad < 0; ++a) {
      for (int b = 0; b <= a; ++b) {
        double v = G[idx[a]][idx[b]] * sc[a] * sc[b];
        for (int c = 0; c < b; ++c) v -= L[a][c] * L[b][c];
        if (!finite_d(v)) {
          bad = a;
          break;
        }
        if (a == b) {
          if (!(v > 1e-10)) {
            bad = a;
            break;
          }
          L[a][a] = sqrt(v);
        } else {
          L[a][b] = v / L[b][b];
        }
      }
    }
    if (bad >= 0) {
      on[idx[bad]] = false;
      continue;
    }
    double y[M], t[M];
    for (int a = 0; a < m; ++a) {
      double v = g[idx[a]] * sc[a];
      for (int c = 0; c < a; ++c) v -= L[a][c] * y[c];
      y[a] = v / L[a][a];
    }
    for (int a = m - 1; a >= 0; --a) {
      double v = y[a];
      for (int c = a + 1; c < m; ++c) v -= L[c][a] * t[c];
      t[a] = v / L[a][a];
    }
    for (int a = 0; a < m; ++a) gamma[idx[a]] = t[a] * sc[a];
    return m;
  }
  return 0;
}

// The 2 x 2 Ritz step of the warm-start correction on the device: dots =
// (p.Ap, p.Ae, e.Ae, p.b, e.b); out = (gamma_p, gamma_e, subspace dim).
__global__ void ritz2_solve_kernel(const double* __restrict__ dots, int use_net, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double full[kRitzSums] = {};
  full[0] = dots[0];                          // G00
  full[1] = dots[1];                          // G01
  full[kRitzVecs] = dots[2];                  // G11
  full[kRitzSums - kRitzVecs] = dots[3];      // g0
  full[kRitzSums - kRitzVecs + 1] = dots[4];  // g1
  const bool use[kRitzVecs] = {true, use_net != 0, false, false};
  double gamma[kRitzVecs];
  const int m = ritz_solve(full, use, gamma);
  out[0] = gamma[0];
  out[1] = gamma[1];
  out[2] = (double)m;
}

template <typename S0, typename SC, typename V>
int learned_solve(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol_factor,
                  int maxit, vflip_solve_stats* stats, const LearnedOpts& lo) {
  const Dims d = T.fine.d;
  const size_t n = d.n();
  int X, Y, Z;
  learned_grid_dims(d.ni, d.nj, d.nk, lo.level, X, Y, Z);
  const size_t nv = (size_t)X * Y * Z;
  float *in2, *out2;
  double* ritz;
  V *x, *r, *r2, *bv, *z, *w0, *w1, *w2, *w3, *q0, *q1, *q2, *q3, *s0, *s1, *q;
  VF_ALLOC(in2, float, "lrn_in2", 2 * nv);
  VF_ALLOC(out2, float, "lrn_out2", 2 * nv);
  VF_ALLOC(ritz, double, "lrn_ritz", kRitzSums);
  VF_ALLOC(x, V, "pcg_x", n);
  VF_ALLOC(r, V, "pcg_r", n);
  VF_ALLOC(z, V, "pcg_z", n);
  VF_ALLOC(s0, V, "pcg_s0", n);
  VF_ALLOC(s1, V, "pcg_s1", n);
  VF_ALLOC(q, V, "pcg_q", n);
  VF_ALLOC(r2, V, "lrn_r2", n);
  VF_ALLOC(bv, V, "lrn_b", n);
  VF_ALLOC(w0, V, "lrn_w0", n);
  VF_ALLOC(w1, V, "lrn_w1", n);
  VF_ALLOC(w2, V, "lrn_w2", n);
  VF_ALLOC(q0, V, "lrn_q0", n);
  VF_ALLOC(q1, V, "lrn_q1", n);
  VF_ALLOC(q2, V, "lrn_q2", n);
  VF_ALLOC(w3, V, "lrn_w3", n);
  VF_ALLOC(q3, V, "lrn_q3", n);
  vflip_learned_stats ls{};
  const bool use_vb = !(lo.mode & VFLIP_LEARNED_NO_VB), use_net = !(lo.mode & VFLIP_LEARNED_NO_NET),
             use_prev = (lo.mode & VFLIP_LEARNED_PREV) != 0;
  const int g = grid_for(n, 256, ctx->num_sms);
  // the incoming pressure (the previous solve's answer) before it is overwritten
  if (use_prev) {
    convert_kernel<V><<<g, 256, 0, ctx->stream>>>(result, w3, n);
    VF_LAUNCH_CHECK();
  } else {
    VF_CUDA(cudaMemsetAsync(w3, 0, n * sizeof(V), ctx->stream));
  }
  int rc;
  VF_CUDA(cudaMemsetAsync(ctx->st, 0, sizeof(PcgScalars), ctx->stream));
  const int gb = grid_for(n, kRedBlock, ctx->num_sms);
  pcg_init_kernel<V, kRedBlock><<<gb, kRedBlock, 0, ctx->stream>>>(rhs, r, x, n, ctx->partials, ctx->st,
                                                                    tol_factor);
  VF_LAUNCH_CHECK();
  if ((rc = read_scalars(ctx))) return rc;
  PcgScalars& h = *ctx->st_host;
  const double rhs_norm = h.res;
  int iterations = 0, vcycles = 0;
  double residual = h.res;
  auto finish = [&](int code) -> int {
    to_double_kernel<V, kRedBlock><<<gb, kRedBlock, 0, ctx->stream>>>(x, result, n);
    ++ctx->launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ctx->fail(VFLIP_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    if (stats) {
      stats->iterations = iterations;
      stats->vcycles = vcycles;
      stats->levels = (int)T.coarse.size() + 1;
      stats->converged = code == VFLIP_OK ? 1 : 0;
      stats->residual = residual;
      stats->rhs_norm = rhs_norm;
    }
    if (lo.lstats) *lo.lstats = ls;
    return code;
  };
  auto fallback = [&]() -> int {
    vflip_solve_stats st2{};
    const int code = pcg_solve(ctx, T, rhs, result, tol_factor, maxit, &st2);
    if (code < 0) return code;
    ls.fallback = 1;
    if (stats) {
      *stats = st2;
      stats->iterations += iterations;
      stats->vcycles += vcycles;
    }
    if (lo.lstats) *lo.lstats = ls;
    return code;
  };
  if (h.res == 0.0) return finish(VFLIP_OK);
  VF_CUDA(cudaMemcpyAsync(bv, r, n * sizeof(V), cudaMemcpyDeviceToDevice, ctx->stream));

  // network: features -> (warm start, coarse correction) on its grid
  float out_scale[2] = {1.0f, 1.0f};
  if (use_net) {
    float* mc;
    double* scale;
    if ((rc = learned_features(ctx, lo, d, rhs, X, Y, Z, in2, &mc, &scale))) return rc;
    vflip::unet::Net& net = *lo.net;
    out_scale[0] = net.out_scale[0];
    out_scale[1] = net.out_scale[1];
    const cudaStream_t saved = net.stream;
    net.stream = ctx->stream;
    cudaEvent_t na, nb;
    VF_CUDA(cudaEventCreate(&na));
    VF_CUDA(cudaEventCreate(&nb));
    cudaEventRecord(na, ctx->stream);
    rc = net.forward_replay(X, Y, Z, in2, out2);
    cudaEventRecord(nb, ctx->stream);
    if (!rc) rc = net.sync_error();
    net.stream = saved;
    if (!rc) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, na, nb);
      ls.net_ms = ms;
    }
    cudaEventDestroy(na);
    cudaEventDestroy(nb);
    if (rc) return ctx->fail(rc, "network: %s", net.err.c_str());
    prolong_trilinear_kernel<V><<<g, 256, 0, ctx->stream>>>(out2, 0, X, Y, Z, lo.level, scale, out_scale[0],
                                                            lo.diag, w1, d.ni, d.nj, d.nk);
    VF_LAUNCH_CHECK();
    prolong_trilinear_kernel<V><<<g, 256, 0, ctx->stream>>>(out2, 1, X, Y, Z, lo.level, scale, out_scale[1],
                                                            lo.diag, w2, d.ni, d.nj, d.nk);
    VF_LAUNCH_CHECK();
  } else {
    VF_CUDA(cudaMemsetAsync(w1, 0, n * sizeof(V), ctx->stream));
    VF_CUDA(cudaMemsetAsync(w2, 0, n * sizeof(V), ctx->stream));
  }

  // initial subspace on the fine grid
  if (use_vb) {
    if ((rc = vcycle<S0, SC, V>(ctx, T, bv, w0, false))) return rc;
    ++vcycles;
  } else {
    VF_CUDA(cudaMemsetAsync(w0, 0, n * sizeof(V), ctx->stream));
  }
  const Level<S0, V>& F = T.fine;
  // the coarse correction corrects V(b); smoothing sweeps on A x = b damp
  // the rough error the coarse prediction and its interpolation carry
  const int ksw = (lo.mode >> 8) & 15;
  if (use_net) {
    vec_add_kernel<V><<<g, 256, 0, ctx->stream>>>(w2, w0, n);
    VF_LAUNCH_CHECK();
  }
  if (use_net && ksw > 0) {
    V* tmp;
    VF_ALLOC(tmp, V, "lrn_tmp", n);
    for (V* v : {w1, w2}) {
      V *src = v, *dst = tmp;
      for (int k = 0; k < ksw; ++k) {
        if ((rc = sweep<S0, V>(ctx, F, bv, src, dst, nullptr, nullptr, nullptr))) return rc;
        std::swap(src, dst);
      }
      if (src != v) VF_CUDA(cudaMemcpyAsync(v, src, n * sizeof(V), cudaMemcpyDeviceToDevice, ctx->stream));
    }
  }
  RitzVecs<V> rv;
  V* ws[kRitzVecs] = {w0, w1, w2, w3};
  V* qs[kRitzVecs] = {q0, q1, q2, q3};
  const bool use[kRitzVecs] = {use_vb, use_net, use_net, use_prev};
  for (int a = 0; a < kRitzVecs; ++a) {
    rv.w[a] = ws[a];
    rv.q[a] = qs[a];
    if (use[a]) {
      spmv_kernel<S0, V><<<g, 256, 0, ctx->stream>>>(ws[a], qs[a], F.diag, F.xp, F.yp, F.zp, d.ni, d.nj, d.nk);
      VF_LAUNCH_CHECK();
    } else {
      VF_CUDA(cudaMemsetAsync(qs[a], 0, n * sizeof(V), ctx->stream));
    }
  }
  const int rb = std::min(gb, kMaxPartials / kRitzSums);
  ritz_dots_kernel<V, kRedBlock><<<rb, kRedBlock, 0, ctx->stream>>>(rv, bv, n, ctx->partials);
  VF_LAUNCH_CHECK();
  ritz_fold_kernel<kRedBlock><<<1, kRedBlock, 0, ctx->stream>>>(ctx->partials, rb, ritz);
  VF_LAUNCH_CHECK();
  double dots[kRitzSums];
  VF_CUDA(cudaMemcpyAsync(dots, ritz, sizeof dots, cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  ls.subspace = ritz_solve(dots, use, ls.gamma);
  for (int a = 0; a < kRitzVecs; ++a) rv.gamma[a] = ls.gamma[a];
  ritz_combine_kernel<V, kRedBlock><<<gb, kRedBlock, 0, ctx->stream>>>(rv, bv, x, r, n, ctx->partials, ctx->st);
  VF_LAUNCH_CHECK();
  if ((rc = read_scalars(ctx))) return rc;
  residual = ls.init_residual = h.res;
  iterations = 1;
  if (h.converged) return finish(VFLIP_OK);
  if (!std::isfinite(h.res)) return fallback();

  // flexible PCG from x0 (Polak-Ribiere beta)
  if ((rc = vcycle<S0, SC, V>(ctx, T, r, z, true))) return rc;
  ++vcycles;
  if ((rc = read_scalars(ctx))) return rc;
  if (h.bad_rho) return fallback();
  V* s_old = s0;
  V* s_new = s1;
  std::vector<double> hist{h.res};
  for (int it = 0; it < maxit; ++it) {
    if ((rc = launch_spmv_dot<V>(ctx, ctx->stream, it == 0, z, s_old, s_new, q, F.diag, F.xp, F.yp, F.zp, d)))
      return rc;
    fcg_update_kernel<V, kRedBlock><<<gb, kRedBlock, 0, ctx->stream>>>(x, r, r2, s_new, q, n, ctx->partials,
                                                                        ctx->st);
    VF_LAUNCH_CHECK();
    if ((rc = read_scalars(ctx))) return rc;
    residual = h.res;
    ++iterations;
    hist.push_back(h.res);
    if (h.converged) return finish(VFLIP_OK);
    const size_t k = hist.size() - 1;
    if (!std::isfinite(h.res) || (k >= 2 && h.res > 0.5 * hist[k - 2])) return fallback();
    std::swap(r, r2);  // r: new residual, r2: previous one
    if ((rc = vcycle<S0, SC, V>(ctx, T, r, z, true))) return rc;
    ++vcycles;
    dot_kernel<V, kRedBlock><<<gb, kRedBlock, 0, ctx->stream>>>(z, r2, n, ctx->partials, ctx->st, kReduceFlex);
    VF_LAUNCH_CHECK();
    std::swap(s_old, s_new);
  }
  return fallback();
}

// ---- the warm-start correction (VFLIP_LEARNED_RESID).  The previous
// pressure p (the result array on entry) is the warm start; the network maps
// its residual r0 = b - A p (features on the level-L grid) to a correction e
// of p; a Ritz step takes x0 = g0 p + g1 e with the energy-optimal g, and
// PCG with the plain V-cycle continues from x0 to |r|_inf <= tol |b|_inf (the
// outer vectors in FP64).  Without the network (NO_NET) the Ritz step scales
// p alone.  A solve that does not converge is repeated by plain MGPCG from
// zero.
template <typename S0, typename SC, typename V>
int learned_resid_prep(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol_factor,
                       OuterVecs<double, V>& o, double** pp_out, double** q1_out) {
  const Dims d = T.fine.d;
  const size_t n = d.n();
  int rc;
  if ((rc = outer_vecs<double>(ctx, T, result, o))) return rc;
  double *pp, *q1;
  VF_ALLOC(pp, double, "lrn_pp", n);
  VF_ALLOC(q1, double, "lrn_q1", n);
  const int g = grid_for(n, 256, ctx->num_sms);
  VF_CUDA(cudaMemcpyAsync(pp, result, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  VF_CUDA(cudaMemsetAsync(ctx->st, 0, sizeof(PcgScalars), ctx->stream));
  launch_pcg_init(ctx, ctx->stream, o, rhs, n, tol_factor);  // r = b, x = 0, tolerance from |b|
  VF_LAUNCH_CHECK();
  spmv_kernel<double, double><<<g, 256, 0, ctx->stream>>>(pp, q1, T.d64, T.x64, T.y64, T.z64, d.ni, d.nj, d.nk);
  VF_LAUNCH_CHECK();
  resid_sub_kernel<V><<<g, 256, 0, ctx->stream>>>(o.r, q1, o.rv, n);  // r0 = b - A p
  VF_LAUNCH_CHECK();
  *pp_out = pp;
  *q1_out = q1;
  return VFLIP_OK;
}

template <typename S0, typename SC, typename V>
int learned_resid_solve(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol_factor,
                        int maxit, vflip_solve_stats* stats, const LearnedOpts& lo) {
  const Dims d = T.fine.d;
  const size_t n = d.n();
  int rc;
  OuterVecs<double, V> o;
  double *pp, *q1;
  if ((rc = learned_resid_prep(ctx, T, rhs, result, tol_factor, o, &pp, &q1))) return rc;
  vflip_learned_stats ls{};
  const bool use_net = !(lo.mode & VFLIP_LEARNED_NO_NET);
  const int g = grid_for(n, 256, ctx->num_sms);
  double *e, *q2, *dots;
  VF_ALLOC(e, double, "lrn_e", n);
  VF_ALLOC(q2, double, "lrn_q2", n);
  VF_ALLOC(dots, double, "lrn_dots", 8);
  if (use_net) {
    int X, Y, Z;
    learned_grid_dims(d.ni, d.nj, d.nk, lo.level, X, Y, Z);
    const size_t nv = (size_t)X * Y * Z;
    float *in2, *out2, *mc;
    double* scale;
    V *ev, *et;
    VF_ALLOC(in2, float, "lrn_in2", 2 * nv);
    VF_ALLOC(out2, float, "lrn_out2", 2 * nv);
    VF_ALLOC(ev, V, "lrn_ev", n);
    VF_ALLOC(et, V, "lrn_et", n);
    if ((rc = learned_features(ctx, lo, d, o.r, X, Y, Z, in2, &mc, &scale))) return rc;
    vflip::unet::Net& net = *lo.net;
    const cudaStream_t saved = net.stream;
    net.stream = ctx->stream;
    cudaEvent_t na, nb;
    VF_CUDA(cudaEventCreate(&na));
    VF_CUDA(cudaEventCreate(&nb));
    cudaEventRecord(na, ctx->stream);
    rc = net.forward_replay(X, Y, Z, in2, out2);
    cudaEventRecord(nb, ctx->stream);
    if (!rc) rc = net.sync_error();
    net.stream = saved;
    if (!rc) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, na, nb);
      ls.net_ms = ms;
    }
    cudaEventDestroy(na);
    cudaEventDestroy(nb);
    if (rc) return ctx->fail(rc, "network: %s", net.err.c_str());
    prolong_trilinear_kernel<V><<<g, 256, 0, ctx->stream>>>(out2, 0, X, Y, Z, lo.level, scale, net.out_scale[0],
                                                            T.d64, ev, d.ni, d.nj, d.nk);
    VF_LAUNCH_CHECK();
    // red-black sweeps on A e = r0 damp the rough error of the interpolated prediction
    const int ksw = (lo.mode >> 8) & 15;
    V *src = ev, *dst = et;
    for (int k = 0; k < ksw; ++k) {
      if ((rc = sweep<S0, V>(ctx, T.fine, o.rv, src, dst, nullptr, nullptr, nullptr))) return rc;
      std::swap(src, dst);
    }
    to_double_kernel<V, kRedBlock><<<grid_for(n, kRedBlock, ctx->num_sms), kRedBlock, 0, ctx->stream>>>(src, e, n);
    VF_LAUNCH_CHECK();
    spmv_kernel<double, double><<<g, 256, 0, ctx->stream>>>(e, q2, T.d64, T.x64, T.y64, T.z64, d.ni, d.nj, d.nk);
    VF_LAUNCH_CHECK();
  } else {
    VF_CUDA(cudaMemsetAsync(e, 0, n * sizeof(double), ctx->stream));
    VF_CUDA(cudaMemsetAsync(q2, 0, n * sizeof(double), ctx->stream));
  }
  const int rb = std::min(grid_for(n, kRedBlock, ctx->num_sms), kMaxPartials / 5);
  ritz2_dots_kernel<kRedBlock><<<rb, kRedBlock, 0, ctx->stream>>>(pp, q1, e, q2, rhs, n, ctx->partials);
  VF_LAUNCH_CHECK();
  ritz2_fold_kernel<kRedBlock><<<1, kRedBlock, 0, ctx->stream>>>(ctx->partials, rb, dots);
  VF_LAUNCH_CHECK();
  // the Ritz step and the combination stay on the device (no host round trip)
  ritz2_solve_kernel<<<1, 32, 0, ctx->stream>>>(dots, use_net ? 1 : 0, dots + 5);
  VF_LAUNCH_CHECK();
  ritz2_combine_kernel<V, kRedBlock><<<grid_for(n, kRedBlock, ctx->num_sms), kRedBlock, 0, ctx->stream>>>(
      pp, q1, e, q2, rhs, dots + 5, o.x, o.r, o.rv, n, ctx->partials, ctx->st);
  VF_LAUNCH_CHECK();
  // the initial residual, kept for the statistics before the loop overwrites it
  VF_CUDA(cudaMemcpyAsync(dots + 3, &ctx->st->res, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  vflip_solve_stats st2{};
  rc = pcg_solve_w<double>(ctx, T, rhs, result, tol_factor, maxit, &st2, (V*)nullptr, true);
  if (rc < 0) return rc;
  double h4[5];
  VF_CUDA(cudaMemcpyAsync(h4, dots + 3, sizeof h4, cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  ls.init_residual = h4[0];
  ls.gamma[0] = h4[2];
  ls.gamma[1] = h4[3];
  ls.subspace = (int)h4[4];
  if (rc != VFLIP_OK) {  // plain MGPCG from zero decides
    vflip_solve_stats st3{};
    const int code = pcg_solve(ctx, T, rhs, result, tol_factor, maxit, &st3);
    if (code < 0) return code;
    ls.fallback = 1;
    st3.iterations += st2.iterations;
    st3.vcycles += st2.vcycles;
    st2 = st3;
    rc = code;
  }
  if (stats) *stats = st2;
  if (lo.lstats) *lo.lstats = ls;
  return rc;
}

// Training triple of the warm-start correction: features of r0 = b - A p
// (p the previous pressure, the result on entry), target R^L (p_new - p) in
// both output channels, weight R^L fluid; the projection itself is plain
// MGPCG (the same answer as without capture).
template <typename S0, typename SC, typename V>
int learned_resid_capture(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol,
                          int maxit, vflip_solve_stats* stats, const LearnedOpts& lo) {
  const Dims d = T.fine.d;
  const size_t n = d.n();
  int rc;
  OuterVecs<double, V> o;
  double *pp, *q1, *r0;
  if ((rc = learned_resid_prep(ctx, T, rhs, result, tol, o, &pp, &q1))) return rc;
  VF_ALLOC(r0, double, "lrn_r0", n);
  VF_CUDA(cudaMemcpyAsync(r0, o.r, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  const int status = pcg_solve(ctx, T, rhs, result, tol, maxit, stats);
  if (status < 0) return status;
  int X, Y, Z;
  learned_grid_dims(d.ni, d.nj, d.nk, lo.level, X, Y, Z);
  const size_t nv = (size_t)X * Y * Z;
  float *mc, *pc;
  double* scale;
  if ((rc = learned_features(ctx, lo, d, r0, X, Y, Z, lo.s_in2, &mc, &scale))) return rc;
  VF_ALLOC(pc, float, "lrn_pc", nv);
  const int gv = grid_for(nv, 256, ctx->num_sms);
  block_average_kernel<double, double><<<gv, 256, 0, ctx->stream>>>(result, pp, 2, d.ni, d.nj, d.nk, lo.level, pc,
                                                                     X, Y, Z);
  VF_LAUNCH_CHECK();
  pack2_kernel<<<gv, 256, 0, ctx->stream>>>(pc, pc, scale, 1, lo.s_tgt2, nv);
  VF_LAUNCH_CHECK();
  VF_CUDA(cudaMemcpyAsync(lo.s_w, mc, nv * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  return status;
}

int check_dims(vflip_ctx* ctx, int ni, int nj, int nk) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (ni <= 0 || nj <= 0 || nk <= 0) return ctx->fail(VFLIP_ERR_ARG, "grid dimensions must be positive");
  // element offsets inside kernels are 32-bit for the face grids too
  if ((double)(ni + 1) * (nj + 1) * (nk + 1) > 2147483647.0) return ctx->fail(VFLIP_ERR_ARG, "grid too large");
  return VFLIP_OK;
}

template <typename S0, typename SC, typename V>
int solve_typed(vflip_ctx* ctx, Typed<S0, SC, V>& T, const double* rhs, double* result, double tol, int maxit,
                vflip_solve_stats* stats, const LearnedOpts* lo) {
  if (lo && (lo->mode & VFLIP_LEARNED_RESID)) {
    if (!std::is_same<V, double>::value && ctx->cfg.pcg_vectors != 0)
      return ctx->fail(VFLIP_ERR_ARG, "the residual mode runs with FP64 PCG vectors (pcg_vectors = 0)");
    if (lo->mode & VFLIP_LEARNED_SOLVE) return learned_resid_solve(ctx, T, rhs, result, tol, maxit, stats, *lo);
    return learned_resid_capture(ctx, T, rhs, result, tol, maxit, stats, *lo);
  }
  if (lo && (lo->mode & VFLIP_LEARNED_SOLVE)) return learned_solve(ctx, T, rhs, result, tol, maxit, stats, *lo);
  if (lo && (lo->mode & VFLIP_LEARNED_CAPTURE)) {
    V* x1;
    VF_ALLOC(x1, V, "lrn_x1", T.fine.d.n());
    const int status = pcg_solve(ctx, T, rhs, result, tol, maxit, stats, x1);
    if (status < 0) return status;
    const int rc = learned_capture<V>(ctx, *lo, T.fine.d, rhs, result, x1);
    return rc ? rc : status;
  }
  return pcg_solve(ctx, T, rhs, result, tol, maxit, stats);
}

int solve_stencil(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp, const double* yp,
                  const double* zp, const double* rhs, double* result, double tol, int maxit,
                  vflip_solve_stats* stats, const LearnedOpts* lo = nullptr) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!diag || !xp || !yp || !zp || !rhs || !result) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  if (maxit < 0) return ctx->fail(VFLIP_ERR_ARG, "max_iterations < 0");
  VF_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  ctx->prof_fine_n = (size_t)ni * nj * nk;
  Hierarchy64 H;
  if ((rc = build_hierarchy64(ctx, ni, nj, nk, diag, xp, yp, zp, H))) return rc;
  int status;
  switch (ctx->cfg.precision) {
    case VFLIP_PREC_FP64: {
      Typed<double, double, double> T;
      if ((rc = make_typed(ctx, H, diag, xp, yp, zp, T, "f64"))) return rc;
      status = solve_typed(ctx, T, rhs, result, tol, maxit, stats, lo);
      break;
    }
    case VFLIP_PREC_FP32: {
      Typed<float, float, float> T;
      if ((rc = make_typed(ctx, H, diag, xp, yp, zp, T, "f32"))) return rc;
      status = solve_typed(ctx, T, rhs, result, tol, maxit, stats, lo);
      break;
    }
    case VFLIP_PREC_MIXED: {
      Typed<float, __nv_bfloat16, float> T;
      if ((rc = make_typed(ctx, H, diag, xp, yp, zp, T, "mix"))) return rc;
      status = solve_typed(ctx, T, rhs, result, tol, maxit, stats, lo);
      break;
    }
    default:
      return ctx->fail(VFLIP_ERR_ARG, "unknown precision %d", ctx->cfg.precision);
  }
  if (status < 0) return status;
  VF_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  VF_CUDA(cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  if (stats) stats->solve_ms = ms;
  return status;
}

// ---------------------------------------------------------------- batched
// Per-system state of a graph-resident batched solve; each system owns a
// sub-context (its scalars, partials, buffers, error flag).
template <typename S0, typename SC, typename V>
struct BatchItem {
  vflip_ctx* sub = nullptr;
  Hierarchy64 H;
  Typed<S0, SC, V> T;
  V *x, *r, *z, *s, *q, *sd;
  int* it;
  cudaGraphConditionalHandle h;
};

int batch_sub(vflip_ctx* ctx, size_t i, vflip_ctx** out) {
  while (ctx->subs.size() <= i) {
    vflip_config c = ctx->cfg;
    c.stream = nullptr;
    vflip_ctx* sub = nullptr;
    const int rc = vflip_create(&sub, &c);
    if (rc) return ctx->fail(rc, "cannot create a per-system context");
    ctx->subs.push_back(sub);
  }
  *out = ctx->subs[i];
  return VFLIP_OK;
}

// Every system's PCG loop as one CUDA graph: per system a parallel branch
// [init] -> while(not converged) {V-cycle; s = z + beta s; q = A s; x, r
// update; condition} -> [FP64 result].  The loop never returns to the host.
template <typename S0, typename SC, typename V>
int batched_graph(vflip_ctx* ctx, int nsys, const vflip_system* sys, double tol, int maxit, vflip_solve_stats* stats,
                  const char* tag) {
  int rc;
  std::vector<BatchItem<S0, SC, V>> items(nsys);
  cudaStream_t cs = nullptr;
  VF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto& it : items)
      if (it.sub) it.sub->stream = nullptr;
    cudaStreamDestroy(cs);
  };
  auto bail = [&](int code) {
    cleanup();
    return code;
  };
  // set-up: hierarchies and vectors (eager, on the capture stream)
  for (int i = 0; i < nsys; ++i) {
    BatchItem<S0, SC, V>& b = items[i];
    if ((rc = batch_sub(ctx, i, &b.sub))) return bail(rc);
    vflip_ctx* c = b.sub;
    c->stream = cs;
    c->profiling = false;
    const vflip_system& y = sys[i];
    if ((rc = build_hierarchy64(c, y.ni, y.nj, y.nk, y.diag, y.xp, y.yp, y.zp, b.H)) ||
        (rc = make_typed(c, b.H, y.diag, y.xp, y.yp, y.zp, b.T, tag))) {
      ctx->err = c->err;
      return bail(rc);
    }
    const size_t n = (size_t)y.ni * y.nj * y.nk;
    V** vs[6] = {&b.x, &b.r, &b.z, &b.s, &b.q, &b.sd};
    const char* names[6] = {"bat_x", "bat_r", "bat_z", "bat_s", "bat_q", "bat_sd"};
    for (int k = 0; k < 6; ++k) {
      *vs[k] = (V*)c->buf(names[k], sizeof(V) * n);
      if (!*vs[k]) return bail(ctx->fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for %s", names[k]));
    }
    b.it = (int*)c->buf("bat_it", sizeof(int));
    if (!b.it) return bail(ctx->fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for bat_it"));
  }
  if (cudaStreamSynchronize(cs) != cudaSuccess) return bail(ctx->fail(VFLIP_ERR_CUDA, "set-up failed"));
  // the graph
  if (cudaGraphCreate(&graph, 0) != cudaSuccess) return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaGraphCreate"));
  auto capture_end = [&](cudaGraph_t g) -> int {
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &out);
    if (e != cudaSuccess || out != g) return ctx->fail(VFLIP_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    return VFLIP_OK;
  };
  for (int i = 0; i < nsys; ++i) {
    BatchItem<S0, SC, V>& b = items[i];
    vflip_ctx* c = b.sub;
    const vflip_system& y = sys[i];
    const size_t n = (size_t)y.ni * y.nj * y.nk;
    const int gb = grid_for(n, kRedBlock, c->num_sms);
    if (cudaGraphConditionalHandleCreate(&b.h, graph, 0, 0) != cudaSuccess)
      return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaGraphConditionalHandleCreate"));
    // init branch
    if (cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCaptureToGraph"));
    cudaMemsetAsync(c->st, 0, sizeof(PcgScalars), cs);
    cudaMemsetAsync(b.s, 0, n * sizeof(V), cs);
    pcg_init_kernel<V, kRedBlock><<<gb, kRedBlock, 0, cs>>>(y.rhs, b.r, b.x, n, c->partials, c->st, tol);
    pcg_loop_init_kernel<<<1, 32, 0, cs>>>(c->st, b.it, b.h);
    cudaStreamCaptureStatus cst;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    if (cudaStreamGetCaptureInfo(cs, &cst, nullptr, nullptr, &deps, &ndeps) != cudaSuccess) {
      cudaStreamEndCapture(cs, &graph);
      return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamGetCaptureInfo"));
    }
    std::vector<cudaGraphNode_t> dv(deps, deps + ndeps);
    if ((rc = capture_end(graph))) return bail(rc);
    // the loop
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = b.h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    if (cudaGraphAddNode(&wn, graph, dv.data(), dv.size(), &cp) != cudaSuccess)
      return bail(ctx->fail(VFLIP_ERR_CUDA, "cannot add the while node"));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCaptureToGraph (body)"));
    const Dims d = b.T.fine.d;
    dim3 sblk(kRedBlock);
    const int kz = 8;
    dim3 sgrid((d.ni + 31) / 32, (d.nj + kRedBlock / 32 - 1) / (kRedBlock / 32), (d.nk + kz - 1) / kz);
    int brc = vcycle<S0, SC, V>(c, b.T, b.r, b.z, true);
    pcg_direction_kernel<V><<<grid_for(n, 256, c->num_sms), 256, 0, cs>>>(b.z, b.s, n, c->st);
    pcg_spmv_dot_kernel<V, true, kRedBlock><<<sgrid, sblk, 0, cs>>>(b.s, nullptr, b.sd, b.q, b.T.fine.diag,
                                                                    b.T.fine.xp, b.T.fine.yp, b.T.fine.zp, d.ni,
                                                                    d.nj, d.nk, kz, c->partials, c->st);
    pcg_update_kernel<V, kRedBlock><<<gb, kRedBlock, 0, cs>>>(b.x, b.r, b.s, b.q, n, c->partials, c->st);
    pcg_loop_cond_kernel<<<1, 32, 0, cs>>>(c->st, b.it, maxit, b.h);
    if ((rc = capture_end(body))) return bail(rc);
    if (brc) {
      ctx->err = c->err;
      return bail(brc);
    }
    if ((size_t)sgrid.x * sgrid.y * sgrid.z > (size_t)kMaxPartials)
      return bail(ctx->fail(VFLIP_ERR_ARG, "grid too large"));
    // result
    if (cudaStreamBeginCaptureToGraph(cs, graph, &wn, nullptr, 1, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCaptureToGraph (result)"));
    to_double_kernel<V, kRedBlock><<<gb, kRedBlock, 0, cs>>>(b.x, y.result, n);
    if ((rc = capture_end(graph))) return bail(rc);
  }
  if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
    return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaGraphInstantiate failed"));
  VF_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  if (cudaGraphLaunch(exec, ctx->stream) != cudaSuccess) return bail(ctx->fail(VFLIP_ERR_CUDA, "cudaGraphLaunch"));
  VF_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  if (cudaEventSynchronize(ctx->ev1) != cudaSuccess) return bail(ctx->fail(VFLIP_ERR_CUDA, "batched graph failed"));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->launches += 1;
  int status = VFLIP_OK;
  for (int i = 0; i < nsys; ++i) {
    BatchItem<S0, SC, V>& b = items[i];
    vflip_ctx* c = b.sub;
    PcgScalars h;
    int iters = 0, kerr = 0;
    if (cudaMemcpy(&h, c->st, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&iters, b.it, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&kerr, c->d_error, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return bail(ctx->fail(VFLIP_ERR_CUDA, "reading the batched results failed"));
    if (kerr) {
      cudaMemset(c->d_error, 0, sizeof(int));
      return bail(ctx->fail(VFLIP_ERR_CUDA, "smoother copy pipeline timed out (system %d)", i));
    }
    const bool conv = h.converged != 0;
    if (!conv) status = VFLIP_NOT_CONVERGED;
    if (stats) {
      stats[i].iterations = iters;
      stats[i].vcycles = iters;
      stats[i].levels = (int)b.T.coarse.size() + 1;
      stats[i].converged = conv ? 1 : 0;
      stats[i].residual = h.res;
      stats[i].rhs_norm = tol > 0.0 ? h.tol / tol : 0.0;
      stats[i].solve_ms = ms;
    }
  }
  cleanup();
  return status;
}

// The whole batch as one persistent cooperative kernel (batch_kernels.cuh)
// inside a captured CUDA graph: the hierarchies are built first (eagerly,
// one per-system context each, as in graph mode), then one launch runs every
// system's PCG loop over a (system, level, chunk) work list.  The cells per
// work item and the resident CTAs per SM come from the context's
// configuration (batch_chunk, batch_ctas_per_sm; vflip_b200/tune.py picks
// them per batch).  A batch the kernel does not take (a system with a single
// level or more levels than it holds) is left to graph mode (*taken false).
template <typename S0, typename SC, typename V>
int batched_persistent(vflip_ctx* ctx, int nsys, const vflip_system* sys, double tol, int maxit,
                       vflip_solve_stats* stats, const char* tag, bool* taken) {
  using A = typename Num<V>::Acc;
  *taken = false;
  int rc;
  std::vector<BatchItem<S0, SC, V>> items(nsys);
  std::vector<BatchSys<S0, SC, V>> desc(nsys);
  const int CH = ctx->cfg.batch_chunk > 0 ? ctx->cfg.batch_chunk : 4096;
  int lmax = 0, part_stride = 1, smem_doubles = 1;
  for (int i = 0; i < nsys; ++i) {
    BatchItem<S0, SC, V>& b = items[i];
    if ((rc = batch_sub(ctx, i, &b.sub))) return rc;
    vflip_ctx* c = b.sub;
    c->stream = ctx->stream;
    c->profiling = false;
    const vflip_system& y = sys[i];
    if ((rc = build_hierarchy64(c, y.ni, y.nj, y.nk, y.diag, y.xp, y.yp, y.zp, b.H)) ||
        (rc = make_typed(c, b.H, y.diag, y.xp, y.yp, y.zp, b.T, tag))) {
      ctx->err = c->err;
      return rc;
    }
    const int nl = (int)b.T.coarse.size() + 1;
    if (nl < 2 || nl > kBatchMaxLevels) return VFLIP_OK;  // not taken
    const size_t n = (size_t)y.ni * y.nj * y.nk;
    V** vs[6] = {&b.x, &b.r, &b.z, &b.s, &b.q, &b.sd};
    const char* names[6] = {"bat_x", "bat_r", "bat_z", "bat_s", "bat_q", "bat_z2"};
    for (int k = 0; k < 6; ++k) {
      *vs[k] = (V*)c->buf(names[k], sizeof(V) * n);
      if (!*vs[k]) return ctx->fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for %s", names[k]);
    }
    b.it = (int*)c->buf("bat_it2", 2 * sizeof(int));  // iterations, state
    if (!b.it) return ctx->fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for bat_it2");
    BatchSys<S0, SC, V>& d = desc[i];
    std::memset(&d, 0, sizeof d);
    d.nl = nl;
    // sweep tiles of kBTX x kBTY x kBTZ cells; their staged region (6 arrays
    // over the tile and a two-cell halo) sets the shared memory
    smem_doubles = std::max(smem_doubles, (int)((6 * (size_t)kBRegion * sizeof(A) + 7) / 8));
    const Level<S0, V>& F = b.T.fine;
    d.fine = BatchLevel<S0, V>{F.d.ni, F.d.nj, F.d.nk, F.diag, F.xp, F.yp, F.zp, b.r, b.z, b.sd,
                               (F.d.ni + kBTX - 1) / kBTX, (F.d.nj + kBTY - 1) / kBTY};
    for (int l = 1; l < nl; ++l) {
      const Level<SC, V>& L = b.T.coarse[l - 1];
      d.lv[l] = BatchLevel<SC, V>{L.d.ni, L.d.nj, L.d.nk, L.diag, L.xp, L.yp, L.zp, L.b, L.xa, L.xb,
                                  (L.d.ni + kBTX - 1) / kBTX, (L.d.nj + kBTY - 1) / kBTY};
    }
    d.x = b.x;
    d.s = b.s;
    d.q = b.q;
    d.rhs = y.rhs;
    d.result = y.result;
    d.st = c->st;
    d.it = b.it;
    d.state = b.it + 1;
    d.direct = b.T.direct.on ? 1 : 0;
    d.bw = b.T.direct.bw;
    d.L = b.T.direct.L;
    d.rinv = b.T.direct.rinv;
    d.ok = b.T.direct.ok;
    d.sweeps = ctx->cfg.coarse_sweeps;
    d.tol_factor = tol;
    lmax = std::max(lmax, nl);
    part_stride = std::max(part_stride, (int)((n + CH - 1) / CH));
    const Level<SC, V>& C = b.T.coarse[nl - 2];
    const int nc = C.d.ni * C.d.nj * C.d.nk;
    smem_doubles = std::max(smem_doubles, d.direct ? nc : (int)((2 * (size_t)nc * sizeof(A) + 7) / 8));
  }
  if (smem_doubles > 26 * 1024) return VFLIP_OK;  // plane window over 208 KB (rows of > 1300 cells): not taken
  if (ctx->cfg.pre_sweeps != 4 || ctx->cfg.post_sweeps != 4) return VFLIP_OK;  // the kernel runs V(4,4)
  // work lists: cell items of level 0 for every system and of a coarser
  // level where the system smooths there; restriction items into level l+1
  const size_t tab = (size_t)lmax * (nsys + 1);
  std::vector<int> cell_pre(tab, 0), rest_pre(tab, 0), sweep_pre(tab, 0);
  for (int l = 0; l < lmax; ++l)
    for (int i = 0; i < nsys; ++i) {
      const BatchSys<S0, SC, V>& d = desc[i];
      long long ci = 0, ri = 0, si = 0;
      if (l == 0) ci = ((long long)d.fine.ni * d.fine.nj * d.fine.nk + CH - 1) / CH;
      if (l + 1 < d.nl) {
        ri = ((long long)d.lv[l + 1].ni * d.lv[l + 1].nj * d.lv[l + 1].nk + CH - 1) / CH;
        const int nk_ = l == 0 ? d.fine.nk : d.lv[l].nk;
        si = (long long)(l == 0 ? d.fine.ntx * d.fine.nty : d.lv[l].ntx * d.lv[l].nty) * ((nk_ + kBTZ - 1) / kBTZ);
      }
      const size_t o = (size_t)l * (nsys + 1) + i;
      cell_pre[o + 1] = cell_pre[o] + (int)ci;
      rest_pre[o + 1] = rest_pre[o] + (int)ri;
      sweep_pre[o + 1] = sweep_pre[o] + (int)si;
    }
  for (int i = 0; i < nsys; ++i) part_stride = std::max(part_stride, sweep_pre[i + 1] - sweep_pre[i]);
  const size_t sys_bytes = ((sizeof(BatchSys<S0, SC, V>) * nsys + 255) / 256) * 256;
  const size_t part_bytes = (size_t)nsys * part_stride * sizeof(double);
  char* dev = (char*)ctx->buf("bp_plan", sys_bytes + part_bytes + (3 * tab + 4) * sizeof(int));
  if (!dev) return ctx->fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for the batch plan");
  auto* dsys = reinterpret_cast<BatchSys<S0, SC, V>*>(dev);
  double* part = reinterpret_cast<double*>(dev + sys_bytes);
  int* dcell = reinterpret_cast<int*>(dev + sys_bytes + part_bytes);
  int* drest = dcell + tab;
  int* dsweep = drest + tab;
  int* dactive = dsweep + tab;
  VF_CUDA(cudaMemcpyAsync(dsys, desc.data(), sizeof(BatchSys<S0, SC, V>) * nsys, cudaMemcpyHostToDevice,
                          ctx->stream));
  VF_CUDA(cudaMemcpyAsync(dcell, cell_pre.data(), tab * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  VF_CUDA(cudaMemcpyAsync(drest, rest_pre.data(), tab * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  VF_CUDA(cudaMemcpyAsync(dsweep, sweep_pre.data(), tab * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  // the host vectors above are read by the copies: wait for them before they go
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  BatchPlan plan{nsys, lmax, maxit, CH, dcell, drest, dsweep, part, part_stride, dactive, smem_doubles};
  auto kern = batch_pcg_kernel<S0, SC, V>;
  const size_t smem = (size_t)smem_doubles * sizeof(double);
  if (smem_optin((const void*)kern, (int)smem) != cudaSuccess)
    return ctx->fail(VFLIP_ERR_CUDA, "cannot raise the batch kernel's shared memory limit");
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchThreads, smem) != cudaSuccess || per_sm < 1)
    return ctx->fail(VFLIP_ERR_CUDA, "the batch kernel cannot be resident");
  if (ctx->cfg.batch_ctas_per_sm > 0) per_sm = std::min(per_sm, ctx->cfg.batch_ctas_per_sm);
  const int grid = per_sm * ctx->num_sms;
  // the launch, captured into a graph (a cooperative kernel node) on a private stream
  cudaStream_t cs = nullptr;
  VF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto done = [&](int code) {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    return code;
  };
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(grid);
  lc.blockDim = dim3(kBatchThreads);
  lc.dynamicSmemBytes = smem;
  lc.stream = cs;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return done(ctx->fail(VFLIP_ERR_CUDA, "cudaStreamBeginCapture (batch)"));
  const cudaError_t le = cudaLaunchKernelEx(&lc, kern, (const BatchSys<S0, SC, V>*)dsys, plan);
  const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
  if (le != cudaSuccess || ce != cudaSuccess)
    return done(ctx->fail(VFLIP_ERR_CUDA, "capturing the persistent batch kernel: %s",
                          cudaGetErrorString(le != cudaSuccess ? le : ce)));
  if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
    return done(ctx->fail(VFLIP_ERR_CUDA, "cudaGraphInstantiate (batch)"));
  *taken = true;
  VF_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  if (cudaGraphLaunch(exec, ctx->stream) != cudaSuccess)
    return done(ctx->fail(VFLIP_ERR_CUDA, "cudaGraphLaunch (batch)"));
  VF_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  if (cudaEventSynchronize(ctx->ev1) != cudaSuccess) return done(ctx->fail(VFLIP_ERR_CUDA, "persistent batch failed"));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->launches += 1;
  int status = VFLIP_OK;
  for (int i = 0; i < nsys; ++i) {
    PcgScalars h;
    int itst[2] = {0, 0};
    if (cudaMemcpy(&h, desc[i].st, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(itst, items[i].it, sizeof itst, cudaMemcpyDeviceToHost) != cudaSuccess)
      return done(ctx->fail(VFLIP_ERR_CUDA, "reading the batched results failed"));
    const bool conv = itst[1] == 0 && h.converged != 0;
    if (!conv) status = VFLIP_NOT_CONVERGED;
    if (stats) {
      stats[i].iterations = itst[1] == 2 ? 0 : itst[0];
      stats[i].vcycles = itst[0] + (itst[1] == 2 ? 1 : 0);
      stats[i].levels = desc[i].nl;
      stats[i].converged = conv ? 1 : 0;
      stats[i].residual = h.res;
      stats[i].rhs_norm = h.rhs_norm;
      stats[i].solve_ms = ms;
    }
  }
  return done(status);
}

}  // namespace

// ============================================================== C ABI}  // namespace

// ============================================================== C ABI
extern "C" {

size_t vflip_config_size(void) { return sizeof(vflip_config); }

void vflip_config_default(vflip_config* cfg) {
  if (!cfg) return;
  cfg->precision = VFLIP_PREC_FP32;
  cfg->pre_sweeps = 4;
  cfg->post_sweeps = 4;
  cfg->coarse_sweeps = 0;          // automatic, see vflip_create
  cfg->coarsest_max_unknowns = 0;
  cfg->device = 0;
  cfg->stream = nullptr;
  cfg->sweep_kernel = 0;
  cfg->smoother_depth = 0;
  cfg->smoother_tile_rows = 0;
  cfg->smoother_plane_ranges = 0;
  cfg->smoother_ctas_per_sm = 0;
  cfg->smoother_threads = 0;
  cfg->smoother_prefetch = 0;
  cfg->coarsest_solver = 0;
  cfg->spmv_kernel = 0;
  cfg->pcg_loop = 0;
  cfg->pcg_vectors = 0;
  cfg->batch_chunk = 0;
  cfg->batch_ctas_per_sm = 0;
  cfg->coarse_tail = 0;
  cfg->tile_sweep_max_cells = 0;
  cfg->p2g_kernel = 0;
  cfg->advect_kernel = 0;
}

int vflip_create(vflip_ctx** out, const vflip_config* cfg) {
  if (!out) return VFLIP_ERR_ARG;
  *out = nullptr;
  vflip_ctx* ctx = new vflip_ctx();
  if (cfg) ctx->cfg = *cfg;
  else vflip_config_default(&ctx->cfg);
  auto bad = [&](int code) {
    delete ctx;
    return code;
  };
  // automatic coarse level: FP64 keeps the reference's hierarchy (16^3
  // coarsest level, 200 sweeps: the bit-exact V-cycle); FP32/MIXED coarsen to
  // 8^3, which 100 sweeps solve to convergence (one PCG iteration fewer on the
  // 256^3 plume operator than 200 sweeps on 16^3)
  const bool f64 = ctx->cfg.precision == VFLIP_PREC_FP64;
  // with the FP64 direct solve, FP32/MIXED coarsen on to <= 64 unknowns
  // (4^3): its band factor then sits in shared memory for the solve
  const bool direct = ctx->cfg.coarsest_solver == 2 || (ctx->cfg.coarsest_solver == 0 && !f64);
  if (ctx->cfg.coarse_sweeps == 0) ctx->cfg.coarse_sweeps = f64 ? 200 : 100;
  if (ctx->cfg.coarsest_max_unknowns == 0)
    ctx->cfg.coarsest_max_unknowns = f64 ? 16 * 16 * 16 : (direct ? 4 * 4 * 4 : 8 * 8 * 8);
  if (ctx->cfg.pre_sweeps < 0 || ctx->cfg.post_sweeps < 0 || ctx->cfg.coarse_sweeps < 0 ||
      ctx->cfg.coarsest_max_unknowns < 1 || ctx->cfg.coarsest_max_unknowns > 4096 || ctx->cfg.precision < 0 ||
      ctx->cfg.precision > 2 || ctx->cfg.sweep_kernel < 0 || ctx->cfg.sweep_kernel > 4 ||
      ctx->cfg.smoother_depth < 0 || ctx->cfg.smoother_tile_rows < 0 || ctx->cfg.smoother_plane_ranges < 0 ||
      ctx->cfg.smoother_ctas_per_sm < 0 ||
      (ctx->cfg.smoother_threads != 0 && ctx->cfg.smoother_threads != kTmaBlock &&
       ctx->cfg.smoother_threads != kTmaBlockWide) ||
      ctx->cfg.coarsest_solver < 0 || ctx->cfg.coarsest_solver > 2 || ctx->cfg.spmv_kernel < 0 ||
      ctx->cfg.spmv_kernel > 1 ||
      ctx->cfg.pcg_loop < 0 || ctx->cfg.pcg_loop > 1 || ctx->cfg.pcg_vectors < 0 || ctx->cfg.pcg_vectors > 1 || ctx->cfg.batch_chunk < 0 || ctx->cfg.batch_ctas_per_sm < 0 ||
      ctx->cfg.coarse_tail < 0 || ctx->cfg.coarse_tail > 1 || ctx->cfg.tile_sweep_max_cells < -1 ||
      ctx->cfg.p2g_kernel < 0 || ctx->cfg.p2g_kernel > 3 || ctx->cfg.advect_kernel < 0 ||
      ctx->cfg.advect_kernel > 1)
    return bad(VFLIP_ERR_ARG);
  if (ctx->cfg.tile_sweep_max_cells == 0) ctx->cfg.tile_sweep_max_cells = 64 * 64 * 64;
  if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) return bad(VFLIP_ERR_CUDA);
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->cfg.device);
  // NULL selects the CUDA default stream, so work is ordered with whatever
  // the caller ran on it (e.g. torch's default stream)
  ctx->stream = (cudaStream_t)ctx->cfg.stream;
  if (cudaMalloc(&ctx->st, sizeof(PcgScalars)) != cudaSuccess) return bad(VFLIP_ERR_NOMEM);
  if (cudaMalloc(&ctx->partials, sizeof(double) * kMaxPartials) != cudaSuccess) return bad(VFLIP_ERR_NOMEM);
  if (cudaMalloc(&ctx->d_error, sizeof(int)) != cudaSuccess) return bad(VFLIP_ERR_NOMEM);
  if (cudaMemset(ctx->d_error, 0, sizeof(int)) != cudaSuccess) return bad(VFLIP_ERR_CUDA);
  if (cudaMallocHost(&ctx->st_host, sizeof(PcgScalars)) != cudaSuccess) return bad(VFLIP_ERR_NOMEM);
  if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess)
    return bad(VFLIP_ERR_CUDA);
  *out = ctx;
  return VFLIP_OK;
}

int vflip_destroy(vflip_ctx* ctx) {
  if (!ctx) return VFLIP_ERR_ARG;
  cudaStreamSynchronize(ctx->stream);
  for (vflip_ctx* sub : ctx->subs) vflip_destroy(sub);
  for (auto& g : ctx->pgs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  if (ctx->pg_stream) cudaStreamDestroy(ctx->pg_stream);
  for (auto& kv : ctx->bufs) cudaFree(kv.second.first);
  if (ctx->st) cudaFree(ctx->st);
  if (ctx->partials) cudaFree(ctx->partials);
  if (ctx->d_error) cudaFree(ctx->d_error);
  if (ctx->st_host) cudaFreeHost(ctx->st_host);
  if (ctx->hbuf) cudaFreeHost(ctx->hbuf);
  for (auto& pe : ctx->prof_events) {
    cudaEventDestroy(pe.a);
    cudaEventDestroy(pe.b);
  }
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  delete ctx;
  return VFLIP_OK;
}

const char* vflip_last_error(const vflip_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int vflip_synchronize(vflip_ctx* ctx) {
  if (!ctx) return VFLIP_ERR_ARG;
  int err = 0;
  VF_CUDA(cudaMemcpyAsync(&ctx->st_host->kernel_error, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  err = ctx->st_host->kernel_error;
  return check_kernel_error(ctx, err);
}

double vflip_last_ms(const vflip_ctx* ctx) { return ctx ? ctx->last_ms : 0.0; }

int vflip_amgpcg_solve(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp,
                       const double* yp, const double* zp, const double* rhs, double* result,
                       double tolerance_factor, int max_iterations, vflip_solve_stats* stats) {
  return solve_stencil(ctx, ni, nj, nk, diag, xp, yp, zp, rhs, result, tolerance_factor, max_iterations, stats);
}

int vflip_amgpcg_solve_csr(vflip_ctx* ctx, uint32_t n, const uint32_t* rowstart, const uint32_t* colindex,
                           const double* value, const double* rhs, double* result, double tolerance_factor,
                           int max_iterations, double* residual_out, int* iterations_out, int ni, int nj, int nk) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!rowstart || !colindex || !value || !rhs || !result) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  if ((size_t)n != (size_t)ni * nj * nk) return ctx->fail(VFLIP_ERR_ARG, "n != ni*nj*nk");
  // pinned staging: diag, +x, +y, +z couplings and the rhs, uploaded as one copy
  double* st = (double*)ctx->host_buf(5 * sizeof(double) * (size_t)n);
  if (!st) return ctx->fail(VFLIP_ERR_NOMEM, "cudaMallocHost failed for the CSR staging buffer");
  const long long sy = ni, sz = (long long)ni * nj;
  // pass 1: CSR -> stencil, checking the pattern (no wrap-around across rows
  // or planes); a repeated entry keeps its last value.  Rows are split over
  // host threads; the first bad row in row order is the one reported.
  uint32_t bad_row = csr_rows_parallel(n, [&](uint32_t r) -> bool {
    int i = (int)(r % ni), j = (int)((r / ni) % nj), k = (int)(r / sz);
    double d = 0.0, px = 0.0, py = 0.0, pz = 0.0;
    for (uint32_t e = rowstart[r]; e < rowstart[r + 1]; ++e) {
      long long dlt = (long long)colindex[e] - (long long)r;
      if (dlt == 0) d = value[e];
      else if (dlt == 1 && i < ni - 1) px = value[e];
      else if (dlt == sy && j < nj - 1) py = value[e];
      else if (dlt == sz && k < nk - 1) pz = value[e];
      else if (!((dlt == -1 && i > 0) || (dlt == -sy && j > 0) || (dlt == -sz && k > 0)))
        return false;
    }
    st[r] = d;
    st[(size_t)n + r] = px;
    st[2 * (size_t)n + r] = py;
    st[3 * (size_t)n + r] = pz;
    st[4 * (size_t)n + r] = rhs[r];
    return true;
  });
  if (bad_row != UINT32_MAX) {
    uint32_t col = 0;
    for (uint32_t e = rowstart[bad_row]; e < rowstart[bad_row + 1]; ++e) {
      long long dlt = (long long)colindex[e] - (long long)bad_row;
      int i = (int)(bad_row % ni), j = (int)((bad_row / ni) % nj), k = (int)(bad_row / sz);
      bool ok = dlt == 0 || (dlt == 1 && i < ni - 1) || (dlt == sy && j < nj - 1) || (dlt == sz && k < nk - 1) ||
                (dlt == -1 && i > 0) || (dlt == -sy && j > 0) || (dlt == -sz && k > 0);
      if (!ok) {
        col = colindex[e];
        break;
      }
    }
    return ctx->fail(VFLIP_ERR_NOT_7POINT, "row %u has an entry at column %u off the 7-point pattern", bad_row, col);
  }
  // pass 2, symmetry: the -x coupling of r (0 when absent) equals the +x
  // coupling of r-1, and likewise in y and z
  bad_row = csr_rows_parallel(n, [&](uint32_t r) -> bool {
    int i = (int)(r % ni), j = (int)((r / ni) % nj), k = (int)(r / sz);
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (uint32_t e = rowstart[r]; e < rowstart[r + 1]; ++e) {
      long long dlt = (long long)colindex[e] - (long long)r;
      if (dlt == -1) mx = value[e];
      else if (dlt == -sy) my = value[e];
      else if (dlt == -sz) mz = value[e];
    }
    bool ok = true;
    if (i > 0) ok &= mx == st[(size_t)n + r - 1];
    if (j > 0) ok &= my == st[2 * (size_t)n + r - sy];
    if (k > 0) ok &= mz == st[3 * (size_t)n + r - sz];
    return ok;
  });
  if (bad_row != UINT32_MAX) return ctx->fail(VFLIP_ERR_NOT_SYMMETRIC, "matrix is not symmetric at row %u", bad_row);
  double *dd, *dres;
  VF_ALLOC(dd, double, "csr_op", 5 * (size_t)n);
  VF_ALLOC(dres, double, "csr_res", n);
  VF_CUDA(cudaMemcpyAsync(dd, st, 5 * sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  vflip_solve_stats s{};
  int status = solve_stencil(ctx, ni, nj, nk, dd, dd + n, dd + 2 * (size_t)n, dd + 3 * (size_t)n,
                             dd + 4 * (size_t)n, dres, tolerance_factor, max_iterations, &s);
  if (status < 0) return status;
  VF_CUDA(cudaMemcpyAsync(st, dres, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  csr_rows_parallel(n, [&](uint32_t r) -> bool {
    result[r] = st[r];
    return true;
  });
  if (residual_out) *residual_out = s.residual;
  if (iterations_out) *iterations_out = s.iterations;
  return status;
}

int vflip_build_levels(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp,
                       const double* yp, const double* zp, int max_levels, int* dims_out, double* levels_out) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!diag || !xp || !yp || !zp) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  Hierarchy64 H;
  if ((rc = build_hierarchy64(ctx, ni, nj, nk, diag, xp, yp, zp, H))) return rc;
  int nl = (int)H.dims.size();
  if (dims_out)
    for (int l = 0; l < nl && l < max_levels; ++l) {
      dims_out[3 * l] = H.dims[l].ni;
      dims_out[3 * l + 1] = H.dims[l].nj;
      dims_out[3 * l + 2] = H.dims[l].nk;
    }
  if (levels_out) {
    size_t off = 0;
    for (int l = 0; l < nl && l < max_levels; ++l) {
      size_t n = H.dims[l].n();
      if (l == 0) {
        VF_CUDA(cudaMemcpyAsync(levels_out, diag, 8 * n, cudaMemcpyDeviceToDevice, ctx->stream));
        VF_CUDA(cudaMemcpyAsync(levels_out + n, xp, 8 * n, cudaMemcpyDeviceToDevice, ctx->stream));
        VF_CUDA(cudaMemcpyAsync(levels_out + 2 * n, yp, 8 * n, cudaMemcpyDeviceToDevice, ctx->stream));
        VF_CUDA(cudaMemcpyAsync(levels_out + 3 * n, zp, 8 * n, cudaMemcpyDeviceToDevice, ctx->stream));
      } else {
        VF_CUDA(cudaMemcpyAsync(levels_out + off, H.lv[l], 32 * n, cudaMemcpyDeviceToDevice, ctx->stream));
      }
      off += 4 * n;
    }
  }
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  return nl;
}

int vflip_rbgs(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp, const double* yp,
               const double* zp, const double* b, double* x, int iterations) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!diag || !xp || !yp || !zp || !b || !x || iterations < 0) return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  size_t n = (size_t)ni * nj * nk;
  double* tmp;
  VF_ALLOC(tmp, double, "rbgs_tmp", n);
  Level<double, double> L{{ni, nj, nk}, diag, xp, yp, zp, nullptr, nullptr, nullptr};
  double* cur = x;
  for (int s = 0; s < iterations; ++s) {
    double* out = (cur == x) ? tmp : x;
    if ((rc = sweep<double, double>(ctx, L, b, cur, out, nullptr, nullptr, nullptr))) return rc;
    cur = out;
  }
  if (cur != x) VF_CUDA(cudaMemcpyAsync(x, cur, 8 * n, cudaMemcpyDeviceToDevice, ctx->stream));
  return VFLIP_OK;
}

int vflip_vcycle(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp, const double* yp,
                 const double* zp, const double* b, double* x) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!diag || !xp || !yp || !zp || !b || !x) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  Hierarchy64 H;
  if ((rc = build_hierarchy64(ctx, ni, nj, nk, diag, xp, yp, zp, H))) return rc;
  size_t n = (size_t)ni * nj * nk;
  const int gb = grid_for(n, 256, ctx->num_sms);
  switch (ctx->cfg.precision) {
    case VFLIP_PREC_FP64: {
      Typed<double, double, double> T;
      if ((rc = make_typed(ctx, H, diag, xp, yp, zp, T, "f64"))) return rc;
      return vcycle(ctx, T, b, x, false);
    }
    case VFLIP_PREC_FP32:
    case VFLIP_PREC_MIXED: {
      float *bf, *xf;
      VF_ALLOC(bf, float, "vc_b", n);
      VF_ALLOC(xf, float, "vc_x", n);
      convert_kernel<float><<<gb, 256, 0, ctx->stream>>>(b, bf, n);
      VF_LAUNCH_CHECK();
      if (ctx->cfg.precision == VFLIP_PREC_FP32) {
        Typed<float, float, float> T;
        if ((rc = make_typed(ctx, H, diag, xp, yp, zp, T, "f32"))) return rc;
        if ((rc = vcycle(ctx, T, bf, xf, false))) return rc;
      } else {
        Typed<float, __nv_bfloat16, float> T;
        if ((rc = make_typed(ctx, H, diag, xp, yp, zp, T, "mix"))) return rc;
        if ((rc = vcycle(ctx, T, bf, xf, false))) return rc;
      }
      to_double_kernel<float, 256><<<gb, 256, 0, ctx->stream>>>(xf, x, n);
      VF_LAUNCH_CHECK();
      return VFLIP_OK;
    }
  }
  return ctx->fail(VFLIP_ERR_ARG, "unknown precision");
}

int vflip_face_weights(vflip_ctx* ctx, int ni, int nj, int nk, const float* nodal_phi, float* uw, float* vw,
                       float* ww) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!nodal_phi || !uw || !vw || !ww) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  dim3 blk(32, 8), grid((ni + 1 + 31) / 32, (nj + 1 + 7) / 8, nk + 1);
  face_weights3_kernel<<<grid, blk, 0, ctx->stream>>>(nodal_phi, uw, vw, ww, ni, nj, nk);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

}  // extern "C"

namespace {

// variant 0: SmokeSolver3D::pcg_projection (inflow overwrite, 1/h^2 terms);
// variant 1: SubDomainSolver::pcg_projection (no inflow, dt/h^2 terms)
int assemble_impl(vflip_ctx* ctx, int variant, int ni, int nj, int nk, float h, float dt, float U_in,
                  const float* nodal_phi, const int8_t* bdesc, const float* us, const float* vs, const float* ws,
                  float* u, float* v, float* w, double* diag, double* xp, double* yp, double* zp, double* rhs,
                  float* op32 = nullptr) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!nodal_phi || (variant == 0 && !bdesc) || !us || !vs || !ws || !u || !v || !w || !diag || !xp || !yp || !zp ||
      !rhs)
    return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  size_t nu = (size_t)(ni + 1) * nj * nk, nv = (size_t)ni * (nj + 1) * nk, nw = (size_t)ni * nj * (nk + 1);
  float* wts;
  VF_ALLOC(wts, float, "face_weights", nu + nv + nw);
  if ((rc = vflip_face_weights(ctx, ni, nj, nk, nodal_phi, wts, wts + nu, wts + nu + nv))) return rc;
  size_t n = (size_t)ni * nj * nk;
  if (variant == 0) {
    inflow_kernel<<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(bdesc, u, v, w, U_in, ni, nj, nk);
    VF_LAUNCH_CHECK();
  }
  assemble_kernel<<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(
      u, v, w, wts, wts + nu, wts + nu + nv, us, vs, ws, diag, xp, yp, zp, rhs, h, ni, nj, nk, variant, dt,
      (float)inv_pow2(h), op32);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int project_impl(vflip_ctx* ctx, int variant, int ni, int nj, int nk, float h, float dt, float U_in,
                 const float* nodal_phi, const int8_t* bdesc, const float* us, const float* vs, const float* ws,
                 float* u, float* v, float* w, double* pressure, double tolerance_factor, int max_iterations,
                 vflip_solve_stats* stats, LearnedOpts* lo = nullptr) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  size_t n = (size_t)ni * nj * nk;
  double *op, *rhs, *p;
  VF_ALLOC(op, double, "proj_op", 4 * n);
  VF_ALLOC(rhs, double, "proj_rhs", n);
  if (pressure) p = pressure;
  else VF_ALLOC(p, double, "proj_p", n);
  cudaEvent_t e0;
  VF_CUDA(cudaEventCreate(&e0));
  VF_CUDA(cudaEventRecord(e0, ctx->stream));
  // FP32/MIXED contexts: the assembly also writes the fine level's FP32
  // operator into the buffer the solve's hierarchy uses for it
  float* op32 = nullptr;
  if (ctx->cfg.precision == VFLIP_PREC_FP32 || ctx->cfg.precision == VFLIP_PREC_MIXED) {
    const char* tag = ctx->cfg.precision == VFLIP_PREC_FP32 ? "f32" : "mix";
    VF_ALLOC(op32, float, std::string(tag) + "_op_0", 4 * n);
  }
  if ((rc = assemble_impl(ctx, variant, ni, nj, nk, h, dt, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w, op,
                          op + n, op + 2 * n, op + 3 * n, rhs, op32))) {
    cudaEventDestroy(e0);
    return rc;
  }
  vflip_solve_stats s{};
  if (lo) lo->diag = op;
  ctx->offdiag_f32 = true;  // assemble_kernel writes every coupling as (double) of a float
  ctx->fine_op_ready = op32;
  int status = solve_stencil(ctx, ni, nj, nk, op, op + n, op + 2 * n, op + 3 * n, rhs, p, tolerance_factor,
                             max_iterations, &s, lo);
  ctx->offdiag_f32 = false;
  ctx->fine_op_ready = nullptr;
  if (status < 0) {
    cudaEventDestroy(e0);
    return status;
  }
  size_t nu = (size_t)(ni + 1) * nj * nk, nv = (size_t)ni * (nj + 1) * nk, nw = (size_t)ni * nj * (nk + 1);
  float* wts = (float*)ctx->buf("face_weights", sizeof(float) * (nu + nv + nw));
  gradient3_kernel<double><<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(
      p, u, v, w, wts, wts + nu, wts + nu + nv, us, vs, ws, h, ni, nj, nk, variant, dt, (float)inv_pow2(h));
  ++ctx->launches;
  cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) {
    cudaEventDestroy(e0);
    return ctx->fail(VFLIP_ERR_CUDA, "launch: %s", cudaGetErrorString(le));
  }
  VF_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  VF_CUDA(cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, ctx->ev1);
  cudaEventDestroy(e0);
  ctx->last_ms = ms;
  if (stats) {
    *stats = s;
    stats->solve_ms = ms;
  }
  return status;
}

}  // namespace

extern "C" {

int vflip_assemble(vflip_ctx* ctx, int ni, int nj, int nk, float h, float U_in, const float* nodal_phi,
                   const int8_t* bdesc, const float* us, const float* vs, const float* ws, float* u, float* v,
                   float* w, double* diag, double* xp, double* yp, double* zp, double* rhs) {
  return assemble_impl(ctx, 0, ni, nj, nk, h, 1.0f, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w, diag, xp, yp, zp,
                       rhs);
}

int vflip_project_subdomain(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* nodal_phi,
                            const float* us, const float* vs, const float* ws, float* u, float* v, float* w,
                            double* pressure, double tolerance_factor, int max_iterations,
                            vflip_solve_stats* stats) {
  return project_impl(ctx, 1, ni, nj, nk, h, dt, 0.0f, nodal_phi, nullptr, us, vs, ws, u, v, w, pressure,
                      tolerance_factor, max_iterations, stats);
}

int vflip_project(vflip_ctx* ctx, int ni, int nj, int nk, float h, float U_in, const float* nodal_phi,
                  const int8_t* bdesc, const float* us, const float* vs, const float* ws, float* u, float* v,
                  float* w, double* pressure, double tolerance_factor, int max_iterations,
                  vflip_solve_stats* stats) {
  return project_impl(ctx, 0, ni, nj, nk, h, 1.0f, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w, pressure,
                      tolerance_factor, max_iterations, stats);
}

int vflip_batched_solve(vflip_ctx* ctx, int nsys, const vflip_system* systems, double tolerance_factor,
                        int max_iterations, int mode, vflip_solve_stats* stats) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (nsys < 0 || (nsys > 0 && !systems)) return ctx->fail(VFLIP_ERR_ARG, "bad system list");
  if (max_iterations < 1) return ctx->fail(VFLIP_ERR_ARG, "max_iterations < 1");
  int rc;
  for (int i = 0; i < nsys; ++i) {
    const vflip_system& y = systems[i];
    if ((rc = check_dims(ctx, y.ni, y.nj, y.nk))) return rc;
    if (!y.diag || !y.xp || !y.yp || !y.zp || !y.rhs || !y.result)
      return ctx->fail(VFLIP_ERR_ARG, "null pointer in system %d", i);
  }
  if (nsys == 0) return VFLIP_OK;
  if (mode == VFLIP_BATCH_LOOP) {
    int status = VFLIP_OK;
    cudaEvent_t a, b;
    VF_CUDA(cudaEventCreate(&a));
    VF_CUDA(cudaEventCreate(&b));
    cudaEventRecord(a, ctx->stream);
    for (int i = 0; i < nsys; ++i) {
      const vflip_system& y = systems[i];
      rc = solve_stencil(ctx, y.ni, y.nj, y.nk, y.diag, y.xp, y.yp, y.zp, y.rhs, y.result, tolerance_factor,
                         max_iterations, stats ? &stats[i] : nullptr);
      if (rc < 0) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return rc;
      }
      if (rc) status = rc;
    }
    cudaEventRecord(b, ctx->stream);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctx->last_ms = ms;
    if (stats)
      for (int i = 0; i < nsys; ++i) stats[i].solve_ms = ms;
    return status;
  }
  if (mode != VFLIP_BATCH_GRAPH && mode != VFLIP_BATCH_PERSISTENT)
    return ctx->fail(VFLIP_ERR_ARG, "unknown batch mode %d", mode);
  cudaEvent_t a;
  VF_CUDA(cudaEventCreate(&a));
  cudaEventRecord(a, ctx->stream);
  if (mode == VFLIP_BATCH_PERSISTENT && ctx->cfg.precision != VFLIP_PREC_FP64) {
    bool taken = false;
    if (ctx->cfg.precision == VFLIP_PREC_FP32)
      rc = batched_persistent<float, float, float>(ctx, nsys, systems, tolerance_factor, max_iterations, stats, "f32",
                                                   &taken);
    else
      rc = batched_persistent<float, __nv_bfloat16, float>(ctx, nsys, systems, tolerance_factor, max_iterations,
                                                           stats, "mix", &taken);
    if (rc < 0 || taken) {
      if (rc >= 0 && stats) {
        // stats: the whole call, set-up included; vflip_last_ms keeps the kernel's graph launch
        cudaEvent_t b;
        float ms = 0.0f;
        if (cudaEventCreate(&b) == cudaSuccess) {
          cudaEventRecord(b, ctx->stream);
          cudaEventSynchronize(b);
          cudaEventElapsedTime(&ms, a, b);
          cudaEventDestroy(b);
        }
        for (int i = 0; i < nsys; ++i) stats[i].solve_ms = ms;
      }
      cudaEventDestroy(a);
      return rc;
    }
  }
  switch (ctx->cfg.precision) {
    case VFLIP_PREC_FP64:
      rc = batched_graph<double, double, double>(ctx, nsys, systems, tolerance_factor, max_iterations, stats, "f64");
      break;
    case VFLIP_PREC_FP32:
      rc = batched_graph<float, float, float>(ctx, nsys, systems, tolerance_factor, max_iterations, stats, "f32");
      break;
    default:
      rc = batched_graph<float, __nv_bfloat16, float>(ctx, nsys, systems, tolerance_factor, max_iterations, stats,
                                                      "mix");
      break;
  }
  if (rc >= 0 && stats) {
    // stats: the whole call, set-up included, like the loop's timing;
    // vflip_last_ms keeps the graph launch alone
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, ctx->ev1);
    for (int i = 0; i < nsys; ++i) stats[i].solve_ms = ms;
  }
  cudaEventDestroy(a);
  return rc;
}

int vflip_learned_grid(int ni, int nj, int nk, int level, int* X, int* Y, int* Z) {
  if (ni <= 0 || nj <= 0 || nk <= 0 || level < 0 || level > 8 || !X || !Y || !Z) return VFLIP_ERR_ARG;
  learned_grid_dims(ni, nj, nk, level, *X, *Y, *Z);
  return VFLIP_OK;
}

int vflip_project_learned(vflip_ctx* ctx, vflip_unet* net, int mode, int level, int ni, int nj, int nk, float h,
                          float U_in, const float* nodal_phi, const int8_t* bdesc, const float* us, const float* vs,
                          const float* ws, float* u, float* v, float* w, double* pressure, double tolerance_factor,
                          int max_iterations, float* sample_in2, float* sample_target2, float* sample_weight,
                          vflip_solve_stats* stats, vflip_learned_stats* lstats) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (level < 0 || level > 8) return ctx->fail(VFLIP_ERR_ARG, "level %d out of range", level);
  const bool solve = (mode & VFLIP_LEARNED_SOLVE) != 0, capture = (mode & VFLIP_LEARNED_CAPTURE) != 0;
  if (solve == capture) return ctx->fail(VFLIP_ERR_ARG, "mode must select exactly one of CAPTURE and SOLVE");
  if (solve && !(mode & VFLIP_LEARNED_NO_NET) && (!net || !net->net))
    return ctx->fail(VFLIP_ERR_ARG, "learned solve needs a network");
  if (capture && (!sample_in2 || !sample_target2 || !sample_weight))
    return ctx->fail(VFLIP_ERR_ARG, "capture needs the three sample buffers");
  if (solve && net && net->net && net->net->device != ctx->cfg.device)
    return ctx->fail(VFLIP_ERR_ARG, "network and context are on different devices");
  LearnedOpts lo;
  lo.net = net ? net->net : nullptr;
  lo.mode = mode;
  lo.level = level;
  lo.s_in2 = sample_in2;
  lo.s_tgt2 = sample_target2;
  lo.s_w = sample_weight;
  lo.lstats = lstats;
  return project_impl(ctx, 0, ni, nj, nk, h, 1.0f, U_in, nodal_phi, bdesc, us, vs, ws, u, v, w, pressure,
                      tolerance_factor, max_iterations, stats, &lo);
}

namespace {
// The lattice (0..2: u, v, w faces, 3: cell centres) of an ni x nj x nk MAC
// grid that a field of fnx x fny x fnz nodes at grid offsets (ox, oy, oz)
// lies on, or -1.
int node_lattice(int ni, int nj, int nk, int fnx, int fny, int fnz, double ox, double oy, double oz) {
  // (float)i - 0.5f is exact below 2^22
  if (std::max(ni, std::max(nj, nk)) >= (1 << 22)) return -1;
  for (int g = 0; g < 4; ++g)
    if (fnx == ni + (g == 0) && fny == nj + (g == 1) && fnz == nk + (g == 2) && ox == (g == 0 ? 0.5 : 0.0) &&
        oy == (g == 1 ? 0.5 : 0.0) && oz == (g == 2 ? 0.5 : 0.0))
      return g;
  return -1;
}
}  // namespace

int vflip_advect_rk2_linear2(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                             const float* v, const float* w, int fnx, int fny, int fnz, double ox, double oy,
                             double oz, const float* field, float* out, const float* field2, float* out2) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (fnx <= 0 || fny <= 0 || fnz <= 0 || !u || !v || !w || !field || !out)
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if ((size_t)fnx * fny * fnz >= (1ull << 31)) return ctx->fail(VFLIP_ERR_ARG, "field too large");
  if (out == field || out == u || out == v || out == w) return ctx->fail(VFLIP_ERR_ARG, "out aliases an input");
  if (field2 && (!out2 || out2 == field2 || out2 == field || out2 == out || out2 == u || out2 == v || out2 == w ||
                 out == field2))
    return ctx->fail(VFLIP_ERR_ARG, "second output missing or aliased");
  const double ih = inv_pow2(h);
  GridView gu{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0, ih};
  GridView gv{v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0, ih};
  GridView gw{w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5, ih};
  GridView gf{field, fnx, fny, fnz, (double)h, ox, oy, oz, ih};
  GridView gf2{field2, fnx, fny, fnz, (double)h, ox, oy, oz, ih};
  size_t n = (size_t)fnx * fny * fnz;
  const int per_block = 256 * 8;
  const unsigned blocks = (unsigned)((n + per_block - 1) / per_block);
  const int slot = prof_start(ctx, field2 ? VFLIP_PROF_ADVECT_PAIR : VFLIP_PROF_ADVECT_FIELD, ctx->stream);
  if (ctx->cfg.precision == VFLIP_PREC_FP64)
    advect_rk2_kernel<true><<<blocks, 256, 0, ctx->stream>>>(gu, gv, gw, gf, out, gf2, field2 ? out2 : nullptr, h, dt,
                                                           per_block);
  else if (ih != 0.0 && ctx->cfg.advect_kernel == 0 && node_lattice(ni, nj, nk, fnx, fny, fnz, ox, oy, oz) >= 0) {
    // the field lies on a lattice whose nodes the first stage reads directly
    const NodeJobs jobs{{NodeJob{field, out, field2, field2 ? out2 : nullptr}, NodeJob{}, NodeJob{}}};
    advect_rk2_node_kernel<<<blocks, 256, 0, ctx->stream>>>(
        u, v, w, ni, nj, nk, (float)ih, h, dt, jobs, node_lattice(ni, nj, nk, fnx, fny, fnz, ox, oy, oz), 1, per_block);
  } else {
    // sample_linear_f's float transform, computed once
    const float ihf = (float)(ih != 0.0 ? ih : 1.0 / (double)h);
    const GridF ff{field, fnx, fny, fnz, (float)ox, (float)oy, (float)oz};
    const GridF ff2{field2, fnx, fny, fnz, (float)ox, (float)oy, (float)oz};
    advect_rk2_f_kernel<<<blocks, 256, 0, ctx->stream>>>(u, v, w, ni, nj, nk, ihf, gf, ff, out, ff2,
                                                         field2 ? out2 : nullptr, h, dt, per_block);
  }
  prof_stop(ctx, slot, ctx->stream);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_advect_rk2_linear(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                            const float* v, const float* w, int fnx, int fny, int fnz, double ox, double oy,
                            double oz, const float* field, float* out) {
  return vflip_advect_rk2_linear2(ctx, ni, nj, nk, h, dt, u, v, w, fnx, fny, fnz, ox, oy, oz, field, out, nullptr,
                                  nullptr);
}

int vflip_advect_velocity_rk2_linear(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                                     const float* v, const float* w, float* uo, float* vo, float* wo) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!u || !v || !w || !uo || !vo || !wo) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  for (const float* o : {(const float*)uo, (const float*)vo, (const float*)wo})
    if (o == u || o == v || o == w) return ctx->fail(VFLIP_ERR_ARG, "an output aliases the velocity");
  if (uo == vo || uo == wo || vo == wo) return ctx->fail(VFLIP_ERR_ARG, "outputs alias each other");
  const double ih = inv_pow2(h);
  if (ctx->cfg.precision != VFLIP_PREC_FP64 && ctx->cfg.advect_kernel == 0 && ih != 0.0 &&
      node_lattice(ni, nj, nk, ni, nj, nk, 0.0, 0.0, 0.0) == 3) {
    // one launch: blocks 3b, 3b+1, 3b+2 advect run b of u, v and w
    const int per_block = 256 * 8;
    size_t most = 0;
    for (size_t c : {(size_t)(ni + 1) * nj * nk, (size_t)ni * (nj + 1) * nk, (size_t)ni * nj * (nk + 1)})
      most = std::max(most, c);
    const NodeJobs jobs{{NodeJob{u, uo, nullptr, nullptr}, NodeJob{v, vo, nullptr, nullptr},
                         NodeJob{w, wo, nullptr, nullptr}}};
    const int slot = prof_start(ctx, VFLIP_PROF_ADVECT_FIELD, ctx->stream);
    advect_rk2_node_kernel<<<3 * (unsigned)((most + per_block - 1) / per_block), 256, 0, ctx->stream>>>(
        u, v, w, ni, nj, nk, (float)ih, h, dt, jobs, 0, 3, per_block);
    prof_stop(ctx, slot, ctx->stream);
    VF_LAUNCH_CHECK();
    return VFLIP_OK;
  }
  if ((rc = vflip_advect_rk2_linear(ctx, ni, nj, nk, h, dt, u, v, w, ni + 1, nj, nk, 0.5, 0.0, 0.0, u, uo)) ||
      (rc = vflip_advect_rk2_linear(ctx, ni, nj, nk, h, dt, u, v, w, ni, nj + 1, nk, 0.0, 0.5, 0.0, v, vo)) ||
      (rc = vflip_advect_rk2_linear(ctx, ni, nj, nk, h, dt, u, v, w, ni, nj, nk + 1, 0.0, 0.0, 0.5, w, wo)))
    return rc;
  return VFLIP_OK;
}

namespace {
// The three MAC velocity views of an ni x nj x nk grid of spacing h.
void velocity_views(const float* u, const float* v, const float* w, int ni, int nj, int nk, float h, GridView& gu,
                    GridView& gv, GridView& gw) {
  const double ih = inv_pow2(h);
  gu = GridView{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0, ih};
  gv = GridView{v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0, ih};
  gw = GridView{w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5, ih};
}

int launch_cubic_clamp(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u, const float* v,
                       const float* w, const CubicFields& job, int nfields) {
  GridView gu, gv, gw;
  velocity_views(u, v, w, ni, nj, nk, h, gu, gv, gw);
  size_t most = 0;
  for (int f = 0; f < nfields; ++f) most = std::max(most, (size_t)job.f[f].nx * job.f[f].ny * job.f[f].nz);
  const int per_block = 256 * 4;
  const dim3 grid((unsigned)((most + per_block - 1) / per_block), (unsigned)nfields);
  if (ctx->cfg.precision == VFLIP_PREC_FP64)
    advect_cubic_clamp_kernel<true><<<grid, 256, 0, ctx->stream>>>(gu, gv, gw, job, h, dt, per_block);
  else
    advect_cubic_clamp_kernel<false><<<grid, 256, 0, ctx->stream>>>(gu, gv, gw, job, h, dt, per_block);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}
}  // namespace

int vflip_advect_cubic_clamp(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                             const float* v, const float* w, int fnx, int fny, int fnz, double ox, double oy,
                             double oz, const float* field, float* out) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (fnx <= 0 || fny <= 0 || fnz <= 0 || !u || !v || !w || !field || !out)
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if ((size_t)fnx * fny * fnz >= (1ull << 31)) return ctx->fail(VFLIP_ERR_ARG, "field too large");
  if (out == field || out == u || out == v || out == w) return ctx->fail(VFLIP_ERR_ARG, "out aliases an input");
  CubicFields job{};
  job.f[0] = GridView{field, fnx, fny, fnz, (double)h, ox, oy, oz, inv_pow2(h)};
  job.out[0] = out;
  return launch_cubic_clamp(ctx, ni, nj, nk, h, dt, u, v, w, job, 1);
}

int vflip_advect_velocity_cubic_clamp(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                                      const float* v, const float* w, float* u_out, float* v_out, float* w_out) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!u || !v || !w || !u_out || !v_out || !w_out) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  const float* ins[3] = {u, v, w};
  float* outs[3] = {u_out, v_out, w_out};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      if (outs[a] == ins[b] || (a != b && outs[a] == outs[b]))
        return ctx->fail(VFLIP_ERR_ARG, "outputs alias the velocity or each other");
  CubicFields job{};
  velocity_views(u, v, w, ni, nj, nk, h, job.f[0], job.f[1], job.f[2]);
  for (int a = 0; a < 3; ++a) job.out[a] = outs[a];
  return launch_cubic_clamp(ctx, ni, nj, nk, h, dt, u, v, w, job, 3);
}

int vflip_advect_rk3_linear2(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                             const float* v, const float* w, int fnx, int fny, int fnz, double fh, double ox,
                             double oy, double oz, const float* field, float* out, const float* field2,
                             float* out2) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (fnx <= 0 || fny <= 0 || fnz <= 0 || !(fh > 0) || !u || !v || !w || !field || !out)
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if ((size_t)fnx * fny * fnz >= (1ull << 31)) return ctx->fail(VFLIP_ERR_ARG, "field too large");
  if (out == field || out == u || out == v || out == w) return ctx->fail(VFLIP_ERR_ARG, "out aliases an input");
  if (field2 && (!out2 || out2 == field2 || out2 == field || out2 == out || out2 == u || out2 == v || out2 == w ||
                 out == field2))
    return ctx->fail(VFLIP_ERR_ARG, "second output missing or aliased");
  GridView gu, gv, gw;
  velocity_views(u, v, w, ni, nj, nk, h, gu, gv, gw);
  const double ih = inv_pow2(fh);
  GridView gf{field, fnx, fny, fnz, fh, ox, oy, oz, ih};
  GridView gf2{field2, fnx, fny, fnz, fh, ox, oy, oz, ih};
  const size_t n = (size_t)fnx * fny * fnz;
  const int per_block = 256 * 4;
  const unsigned blocks = (unsigned)((n + per_block - 1) / per_block);
  float* o2 = field2 ? out2 : nullptr;
  if (ctx->cfg.precision == VFLIP_PREC_FP64)
    advect_rk3_kernel<true><<<blocks, 256, 0, ctx->stream>>>(gu, gv, gw, gf, out, gf2, o2, dt, per_block);
  else
    advect_rk3_kernel<false><<<blocks, 256, 0, ctx->stream>>>(gu, gv, gw, gf, out, gf2, o2, dt, per_block);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_advect_rk3_linear(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                            const float* v, const float* w, int fnx, int fny, int fnz, double fh, double ox,
                            double oy, double oz, const float* field, float* out) {
  return vflip_advect_rk3_linear2(ctx, ni, nj, nk, h, dt, u, v, w, fnx, fny, fnz, fh, ox, oy, oz, field, out,
                                  nullptr, nullptr);
}

int vflip_gen_heat(vflip_ctx* ctx, int fnx, int fny, int fnz, double fh, float dt, float dens_decay,
                   float temp_decay, float cx, float cy, float cz, float radius, float dens, float heat, float* rho,
                   float* temp) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (fnx <= 0 || fny <= 0 || fnz <= 0 || !(fh > 0) || !rho || !temp || rho == temp)
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  const size_t n = (size_t)fnx * fny * fnz;
  if (n >= (1ull << 31)) return ctx->fail(VFLIP_ERR_ARG, "grid too large");
  HeatSource s{dt, dens_decay, temp_decay, cx, cy, cz, radius, dens, heat};
  gen_heat_kernel<<<grid_for(n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(rho, temp, fnx, fny, fnz, (float)fh,
                                                                              s);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_add_smokeforce(vflip_ctx* ctx, void* particles, int np, int fnx, int fny, int fnz, double fh,
                         const float* rho, const float* temp, float alpha, float beta, float dt) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (np < 0 || (np > 0 && !particles) || fnx <= 0 || fny <= 0 || fnz <= 0 || !(fh > 0) || !rho || !temp)
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if (np == 0) return VFLIP_OK;
  const double ih = inv_pow2(fh);
  GridView gr{rho, fnx, fny, fnz, fh, 0.0, 0.0, 0.0, ih}, gt{temp, fnx, fny, fnz, fh, 0.0, 0.0, 0.0, ih};
  add_smokeforce_kernel<<<grid_for(np, 128, ctx->num_sms * 8), 128, 0, ctx->stream>>>((ParticleRec*)particles, np,
                                                                                     gr, gt, alpha, beta, dt);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_delta(vflip_ctx* ctx, size_t n, const float* after, const float* before, float* delta) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (!after || !before || !delta) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  if (n == 0) return VFLIP_OK;
  delta_kernel<<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(after, before, delta, n);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

static int particle_cells_impl(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                         int* cell_out, SubFrame sf) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (np < 0 || (np > 0 && (!particles || !cell_out))) return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if (np == 0) return VFLIP_OK;
  size_t nc = (size_t)ni * nj * nk;
  int *slot, *count;
  VF_ALLOC(slot, int, "p_slot", np);
  VF_ALLOC(count, int, "p_count", nc + 1);
  VF_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (nc + 1), ctx->stream));
  hash_count_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>(
      (const ParticleRec*)particles, np, ni, nj, nk, h, (float)inv_pow2(h), cell_out, slot, count, sf);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_particle_cells(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                         int* cell_out) {
  return particle_cells_impl(ctx, ni, nj, nk, h, particles, np, cell_out, SubFrame{0.0f, 0.0f, 0.0f, 0});
}

}  // extern "C"

namespace {

// Exclusive scan of n ints (n may be large): tiles, then the tile sums
// recursively.
int exclusive_scan(vflip_ctx* ctx, const int* in, int* out, size_t n, int depth = 0) {
  size_t tiles = (n + kScanTile - 1) / kScanTile;
  int* sums = nullptr;
  if (tiles > 1) {
    VF_ALLOC(sums, int, "scan_sums_" + std::to_string(depth), tiles);
  }
  scan_tiles_kernel<<<(unsigned)tiles, kScanBlock, 0, ctx->stream>>>(in, out, sums, n);
  VF_LAUNCH_CHECK();
  if (tiles > 1) {
    int* pre;
    VF_ALLOC(pre, int, "scan_pre_" + std::to_string(depth), tiles);
    int rc = exclusive_scan(ctx, sums, pre, tiles, depth + 1);
    if (rc) return rc;
    scan_add_kernel<<<(unsigned)tiles, 256, 0, ctx->stream>>>(out, pre, n);
    VF_LAUNCH_CHECK();
  }
  return VFLIP_OK;
}

}  // namespace

// Each bucket of `order` (start[c] .. start[c+1]) into ascending particle
// order: insertion sort of up to 32, a warp's bitonic sort in shared memory
// of up to kBigBucket (the buckets listed by sort_buckets_kernel), heapsort
// beyond.
static int sort_buckets(vflip_ctx* ctx, const int* start, int* order, size_t nc, int np) {
  int* big;
  VF_ALLOC(big, int, "p_big", (size_t)np / 33 + 2);  // [0]: the count; at most np / 33 buckets exceed 32
  VF_CUDA(cudaMemsetAsync(big, 0, sizeof(int), ctx->stream));
  sort_buckets_kernel<<<grid_for(nc, 256, ctx->num_sms), 256, 0, ctx->stream>>>(start, order, (int)nc, big + 1, big);
  VF_LAUNCH_CHECK();
  sort_big_buckets_kernel<<<ctx->num_sms * 6, 32 * kBigWarps, 0, ctx->stream>>>(start, order, big + 1, big);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

// The tiled P2G gather over (ni+1) x (nj+1) x (nk+1) node indices in tiles
// of 8 x 8 x TZ: TZ = 8 one CTA per SM, TZ = 4 two, each with the shared
// memory that residency leaves it; SUB: a subdomain's grid.
template <int TZ, bool SUB>
static int launch_p2g_tile(vflip_ctx* ctx, int ni, int nj, int nk, float h, float ih, const int* start,
                           const float4* spos, const float4* svel, float* u, float* ucoef, float* v, float* vcoef,
                           float* w, float* wcoef) {
  using T = P2gTile<TZ, SUB>;
  int per_sm = 0, per_block = 0;
  VF_CUDA(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->cfg.device));
  VF_CUDA(cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->cfg.device));
  // the runtime reserves 1 KB of each resident CTA's shared memory
  const int smem = std::min(per_block, per_sm / T::ctas_per_sm - 1024) & ~15;
  VF_CUDA(smem_optin((const void*)p2g3_tile_kernel<TZ, SUB>, smem));
  const int cap = p2g_tile_cap<TZ, SUB>(smem);
  if (cap < 1) return ctx->fail(VFLIP_ERR_CUDA, "no shared memory for the tiled P2G");
  const int ntx = (ni + kP2gTX) / kP2gTX, nty = (nj + kP2gTY) / kP2gTY, ntz = (nk + TZ) / TZ;
  const size_t tiles = (size_t)ntx * nty * ntz;
  if (tiles > 0x7fffffff) return ctx->fail(VFLIP_ERR_ARG, "grid too large for the tiled P2G");
  p2g3_tile_kernel<TZ, SUB><<<(unsigned)tiles, T::threads, smem, ctx->stream>>>(
      start, spos, svel, u, ucoef, v, vcoef, w, wcoef, ni, nj, nk, h, ih, ntx, nty, cap);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

extern "C" {

static int p2g_impl(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np, float* u,
              float* ucoef, float* v, float* vcoef, float* w, float* wcoef, SubFrame sf) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (np < 0 || (np > 0 && !particles)) return ctx->fail(VFLIP_ERR_ARG, "bad particle array");
  if ((!u) != (!ucoef) || (!v) != (!vcoef) || (!w) != (!wcoef))
    return ctx->fail(VFLIP_ERR_ARG, "field and coef pointers must be given in pairs");
  size_t nc = (size_t)ni * nj * nk;
  int *cell, *slot, *count, *start, *order;
  float4 *spos, *svel;
  size_t npp = np > 0 ? (size_t)np : 1;
  VF_ALLOC(cell, int, "p_cell", npp);
  VF_ALLOC(slot, int, "p_slot", npp);
  VF_ALLOC(count, int, "p_count", nc + 1);
  VF_ALLOC(start, int, "p_start", nc + 1);
  VF_ALLOC(order, int, "p_order", npp);
  VF_ALLOC(spos, float4, "p_spos", npp);
  VF_ALLOC(svel, float4, "p_svel", npp);
  const int sslot = prof_start(ctx, VFLIP_PROF_P2G_SORT, ctx->stream);
  VF_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (nc + 1), ctx->stream));
  if (np > 0) {
    hash_count_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>(
        (const ParticleRec*)particles, np, ni, nj, nk, h, (float)inv_pow2(h), cell, slot, count, sf);
    VF_LAUNCH_CHECK();
  }
  if ((rc = exclusive_scan(ctx, count, start, nc + 1))) return rc;
  if (np > 0) {
    scatter_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>(cell, slot, start, order, np);
    VF_LAUNCH_CHECK();
    if ((rc = sort_buckets(ctx, start, order, nc, np))) return rc;
    gather_sorted_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>(
        (const ParticleRec*)particles, order, spos, svel, start + nc, sf);
    VF_LAUNCH_CHECK();
  }
  prof_stop(ctx, sslot, ctx->stream);
  if (!u && !v && !w) return VFLIP_OK;
  const float ih = (float)inv_pow2(h);
  const int gslot = prof_start(ctx, VFLIP_PROF_P2G_GATHER, ctx->stream);
  if (sf.sub && ctx->cfg.p2g_kernel != 1) {
    const int rc2 =
        ctx->cfg.p2g_kernel == 3
            ? launch_p2g_tile<4, true>(ctx, ni, nj, nk, h, ih, start, spos, svel, u, ucoef, v, vcoef, w, wcoef)
            : launch_p2g_tile<8, true>(ctx, ni, nj, nk, h, ih, start, spos, svel, u, ucoef, v, vcoef, w, wcoef);
    if (rc2) return rc2;
  } else if (sf.sub) {
    // the 9^3 gathers of the boundary shell and the 3^3 ones of the inner box
    // in separate launches, so that no warp mixes the two
    for (int part : {P2G_SHELL, P2G_INNER}) {
      const size_t nn = p2g_part_size(part, ni, nj, nk);
      if (nn == 0) continue;
      p2g3_kernel<true><<<grid_for(nn, 128, ctx->num_sms * 8), 128, 0, ctx->stream>>>(
          start, spos, svel, u, ucoef, v, vcoef, w, wcoef, ni, nj, nk, h, ih, part);
      VF_LAUNCH_CHECK();
    }
  } else if (ctx->cfg.p2g_kernel != 1) {
    const int rc2 = ctx->cfg.p2g_kernel == 3
                        ? launch_p2g_tile<4, false>(ctx, ni, nj, nk, h, ih, start, spos, svel, u, ucoef, v, vcoef, w,
                                                    wcoef)
                        : launch_p2g_tile<8, false>(ctx, ni, nj, nk, h, ih, start, spos, svel, u, ucoef, v, vcoef, w,
                                                    wcoef);
    if (rc2) return rc2;
  } else {
    const size_t nn = p2g_part_size(P2G_ALL, ni, nj, nk);
    p2g3_kernel<false><<<grid_for(nn, 128, ctx->num_sms * 8), 128, 0, ctx->stream>>>(
        start, spos, svel, u, ucoef, v, vcoef, w, wcoef, ni, nj, nk, h, ih, P2G_ALL);
    VF_LAUNCH_CHECK();
  }
  prof_stop(ctx, gslot, ctx->stream);
  return VFLIP_OK;
}

int vflip_p2g(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np, float* u,
              float* ucoef, float* v, float* vcoef, float* w, float* wcoef) {
  return p2g_impl(ctx, ni, nj, nk, h, particles, np, u, ucoef, v, vcoef, w, wcoef, SubFrame{0.0f, 0.0f, 0.0f, 0});
}

}  // extern "C"

// The device view of a nested subdomain (SubDomainSolver::init, sub_domain.h:161-175:
// bmax = bmin + (nx, ny, nz) h, in float); null `sub` gives an inactive view.
static int make_nest(vflip_ctx* ctx, const vflip_subdomain* sub, Nest* out) {
  *out = Nest{};
  if (!sub) return VFLIP_OK;
  int rc;
  if ((rc = check_dims(ctx, sub->ni, sub->nj, sub->nk))) return rc;
  if (!(sub->h > 0.0f) || !sub->u || !sub->v || !sub->w || !sub->nodal_phi)
    return ctx->fail(VFLIP_ERR_ARG, "bad subdomain (spacing or null grid)");
  const int n[3] = {sub->ni, sub->nj, sub->nk};
  for (int a = 0; a < 3; ++a) {
    out->bmin[a] = sub->bmin[a];
    out->bmax[a] = sub->bmin[a] + (float)n[a] * sub->h;
  }
  out->h = sub->h;
  const double hd = sub->h, ih = inv_pow2(sub->h);
  const int ni = sub->ni, nj = sub->nj, nk = sub->nk;
  out->u = GridView{sub->u, ni + 1, nj, nk, hd, 0.5, 0.0, 0.0, ih};
  out->v = GridView{sub->v, ni, nj + 1, nk, hd, 0.0, 0.5, 0.0, ih};
  out->w = GridView{sub->w, ni, nj, nk + 1, hd, 0.0, 0.0, 0.5, ih};
  out->phi = GridView{sub->nodal_phi, ni + 1, nj + 1, nk + 1, hd, 0.5, 0.5, 0.5, ih};
  return VFLIP_OK;
}

static int advect_flip_impl(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np,
                            const float* u, const float* v, const float* w, const float* nodal_phi, float dt,
                            const vflip_subdomain* sub) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (np < 0 || (np > 0 && !particles) || !u || !v || !w || !nodal_phi) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  Nest nest;
  if ((rc = make_nest(ctx, sub, &nest))) return rc;
  if (np == 0) return VFLIP_OK;
  const double hd = h, ih = inv_pow2(h);
  GridView gu{u, ni + 1, nj, nk, hd, 0.5, 0.0, 0.0, ih}, gv{v, ni, nj + 1, nk, hd, 0.0, 0.5, 0.0, ih},
      gw{w, ni, nj, nk + 1, hd, 0.0, 0.0, 0.5, ih}, gp{nodal_phi, ni + 1, nj + 1, nk + 1, hd, 0.5, 0.5, 0.5, ih};
  const int grid = grid_for(np, 128, ctx->num_sms * 8);
  if (sub)
    advect_flip_kernel<true><<<grid, 128, 0, ctx->stream>>>((ParticleRec*)particles, np, gu, gv, gw, gp, dt, nest);
  else
    advect_flip_kernel<false><<<grid, 128, 0, ctx->stream>>>((ParticleRec*)particles, np, gu, gv, gw, gp, dt, nest);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

extern "C" {

int vflip_advect_flip(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np, const float* u,
                      const float* v, const float* w, const float* nodal_phi, float dt) {
  return advect_flip_impl(ctx, ni, nj, nk, h, particles, np, u, v, w, nodal_phi, dt, nullptr);
}

int vflip_advect_flip_nested(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np,
                             const float* u, const float* v, const float* w, const float* nodal_phi, float dt,
                             const vflip_subdomain* sub) {
  if (ctx && !sub) return ctx->fail(VFLIP_ERR_ARG, "null subdomain");
  return advect_flip_impl(ctx, ni, nj, nk, h, particles, np, u, v, w, nodal_phi, dt, sub);
}

int vflip_halo_select(vflip_ctx* ctx, const void* particles, int np, float h, const vflip_subdomain* sub, void* out,
                      int capacity, int* n_out) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (np < 0 || (np > 0 && !particles) || !sub || !out || !n_out || capacity < 0 || !(h > 0.0f))
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  Nest nest;
  int rc;
  if ((rc = make_nest(ctx, sub, &nest))) return rc;
  int *flag, *pos;
  VF_ALLOC(flag, int, "halo_flag", (size_t)np + 1);
  VF_ALLOC(pos, int, "halo_pos", (size_t)np + 1);
  const float dx = (float)(0.5 * (double)h);  // the reference passes 0.5 * _hx (double) to a float
  halo_flag_kernel<<<grid_for((size_t)np + 1, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      (const ParticleRec*)particles, np, nest, dx, flag);
  VF_LAUNCH_CHECK();
  if ((rc = exclusive_scan(ctx, flag, pos, (size_t)np + 1))) return rc;
  if (np > 0) {
    halo_compact_kernel<<<grid_for(np, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
        (const ParticleRec*)particles, np, flag, pos, (ParticleRec*)out, capacity);
    VF_LAUNCH_CHECK();
  }
  int m = 0;
  VF_CUDA(cudaMemcpyAsync(&m, pos + np, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  *n_out = m;
  if (m > capacity) return ctx->fail(VFLIP_ERR_TOO_LARGE, "%d halo particles exceed the capacity %d", m, capacity);
  return VFLIP_OK;
}

static int reorder_flip_impl(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                       const float* u, const float* v, const float* w, const float* nodal_phi, unsigned seed,
                       void* out, int capacity, int* np_out, SubFrame sf, const vflip_subdomain* sub = nullptr) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (np < 0 || (np > 0 && !particles) || !u || !v || !w || !nodal_phi || !out || !np_out || capacity < 0)
    return ctx->fail(VFLIP_ERR_ARG, "null pointer or negative capacity");
  Nest nest;
  if ((rc = make_nest(ctx, sub, &nest))) return rc;
  const size_t nc = (size_t)ni * nj * nk;
  if (9.0 * (double)nc > 2147483000.0) return ctx->fail(VFLIP_ERR_TOO_LARGE, "grid too large for reseeding");
  const int ntmp = (int)(9 * nc);  // at most 9 particles per cell before the solid filter
  int *cell, *slot, *count, *start, *order, *ocount, *base, *keep, *kpos;
  ParticleRec* tmp;
  const size_t npp = np > 0 ? (size_t)np : 1;
  VF_ALLOC(cell, int, "p_cell", npp);
  VF_ALLOC(slot, int, "p_slot", npp);
  VF_ALLOC(count, int, "p_count", nc + 1);
  VF_ALLOC(start, int, "p_start", nc + 1);
  VF_ALLOC(order, int, "p_order", npp);
  VF_ALLOC(ocount, int, "r_count", nc + 1);
  VF_ALLOC(base, int, "r_base", nc + 1);
  VF_ALLOC(tmp, ParticleRec, "r_tmp", ntmp);
  VF_ALLOC(keep, int, "r_keep", (size_t)ntmp + 1);
  VF_ALLOC(kpos, int, "r_kpos", (size_t)ntmp + 1);
  VF_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (nc + 1), ctx->stream));
  if (np > 0) {
    hash_count_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>(
        (const ParticleRec*)particles, np, ni, nj, nk, h, (float)inv_pow2(h), cell, slot, count, sf);
    VF_LAUNCH_CHECK();
  }
  if ((rc = exclusive_scan(ctx, count, start, nc + 1))) return rc;
  if (np > 0) {
    scatter_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>(cell, slot, start, order, np);
    VF_LAUNCH_CHECK();
    if ((rc = sort_buckets(ctx, start, order, nc, np))) return rc;
  }
  reorder_count_kernel<<<grid_for(nc, 256, ctx->num_sms), 256, 0, ctx->stream>>>(start, ocount, (int)nc, ni, nj,
                                                                                  nk, sf.sub);
  VF_LAUNCH_CHECK();
  if ((rc = exclusive_scan(ctx, ocount, base, nc + 1))) return rc;
  const double hd = h, ih = inv_pow2(h);
  GridView gu{u, ni + 1, nj, nk, hd, 0.5, 0.0, 0.0, ih}, gv{v, ni, nj + 1, nk, hd, 0.0, 0.5, 0.0, ih},
      gw{w, ni, nj, nk + 1, hd, 0.0, 0.0, 0.5, ih}, gp{nodal_phi, ni + 1, nj + 1, nk + 1, hd, 0.5, 0.5, 0.5, ih};
  reorder_write_kernel<<<grid_for(nc, 128, ctx->num_sms * 8), 128, 0, ctx->stream>>>(
      (const ParticleRec*)particles, start, order, base, tmp, ni, nj, nk, h, gu, gv, gw, (uint32_t)seed, sf);
  VF_LAUNCH_CHECK();
  solid_keep_kernel<<<grid_for(ntmp, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(tmp, base + nc, keep, gp, ntmp, sf,
                                                                                    sub ? 1 : 0, nest);
  VF_LAUNCH_CHECK();
  if ((rc = exclusive_scan(ctx, keep, kpos, (size_t)ntmp + 1))) return rc;
  compact_kernel<<<grid_for(ntmp, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(tmp, keep, kpos, base + nc,
                                                                                  (ParticleRec*)out, ntmp, capacity);
  VF_LAUNCH_CHECK();
  // kept count = kpos[total]; total <= ntmp by construction
  int total = 0, kept = 0;
  VF_CUDA(cudaMemcpyAsync(&total, base + nc, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  VF_CUDA(cudaMemcpyAsync(&kept, kpos + total, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  *np_out = kept;
  if (kept > capacity) return ctx->fail(VFLIP_ERR_TOO_LARGE, "reseeded particles (%d) exceed the capacity %d", kept,
                                        capacity);
  return VFLIP_OK;
}

int vflip_reorder_flip(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                       const float* u, const float* v, const float* w, const float* nodal_phi, unsigned seed,
                       void* out, int capacity, int* np_out) {
  return reorder_flip_impl(ctx, ni, nj, nk, h, particles, np, u, v, w, nodal_phi, seed, out, capacity, np_out,
                  SubFrame{0.0f, 0.0f, 0.0f, 0});
}

int vflip_reorder_flip_nested(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                              const float* u, const float* v, const float* w, const float* nodal_phi, unsigned seed,
                              void* out, int capacity, int* np_out, const vflip_subdomain* sub) {
  if (ctx && !sub) return ctx->fail(VFLIP_ERR_ARG, "null subdomain");
  return reorder_flip_impl(ctx, ni, nj, nk, h, particles, np, u, v, w, nodal_phi, seed, out, capacity, np_out,
                           SubFrame{0.0f, 0.0f, 0.0f, 0}, sub);
}

int vflip_sub_reorder_flip(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz,
                           const void* particles, int np, const float* u, const float* v, const float* w,
                           const float* nodal_phi, unsigned seed, void* out, int capacity, int* np_out) {
  return reorder_flip_impl(ctx, ni, nj, nk, h, particles, np, u, v, w, nodal_phi, seed, out, capacity, np_out,
                           SubFrame{bx, by, bz, 1});
}

static int g2p_impl(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np, const float* du,
              const float* dv, const float* dw, const float* un, const float* vn, const float* wn,
              double flip_ratio, SubFrame sf) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (np < 0 || (np > 0 && !particles) || !du || !dv || !dw) return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if (flip_ratio != 1.0 && (!un || !vn || !wn)) return ctx->fail(VFLIP_ERR_ARG, "blend needs u_new/v_new/w_new");
  if (np == 0) return VFLIP_OK;
  const double ih = inv_pow2(h);
  GridView gdu{du, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0, ih};
  GridView gdv{dv, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0, ih};
  GridView gdw{dw, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5, ih};
  GridView gun{un ? un : du, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0, ih};
  GridView gvn{vn ? vn : dv, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0, ih};
  GridView gwn{wn ? wn : dw, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5, ih};
  g2p_kernel<<<grid_for(np, 256, ctx->num_sms), 256, 0, ctx->stream>>>((ParticleRec*)particles, np, gdu, gdv, gdw,
                                                                       gun, gvn, gwn, flip_ratio, sf);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_g2p(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np, const float* du,
              const float* dv, const float* dw, const float* un, const float* vn, const float* wn,
              double flip_ratio) {
  return g2p_impl(ctx, ni, nj, nk, h, particles, np, du, dv, dw, un, vn, wn, flip_ratio,
                  SubFrame{0.0f, 0.0f, 0.0f, 0});
}

int vflip_sub_particle_cells(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz,
                             const void* particles, int np, int* cell_out) {
  return particle_cells_impl(ctx, ni, nj, nk, h, particles, np, cell_out, SubFrame{bx, by, bz, 1});
}

int vflip_sub_p2g(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz,
                  const void* particles, int np, float* u, float* ucoef, float* v, float* vcoef, float* w,
                  float* wcoef) {
  return p2g_impl(ctx, ni, nj, nk, h, particles, np, u, ucoef, v, vcoef, w, wcoef, SubFrame{bx, by, bz, 1});
}

int vflip_sub_g2p(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz, void* particles,
                  int np, const float* du, const float* dv, const float* dw) {
  return g2p_impl(ctx, ni, nj, nk, h, particles, np, du, dv, dw, nullptr, nullptr, nullptr, 1.0,
                  SubFrame{bx, by, bz, 1});
}

}  // extern "C"

namespace {
__global__ void bricks_kernel(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz,
                              bool to_linear) {
  const int bx = (nx + 7) / 8, by = (ny + 7) / 8;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    unsigned i = (unsigned)(e % nx), j = (unsigned)((e / nx) % ny), k = (unsigned)(e / ((size_t)nx * ny));
    size_t b = ((size_t)((k >> 3) * bx * by + (j >> 3) * bx + (i >> 3)) << 9) + ((k & 7) << 6) + ((j & 7) << 3) +
               (i & 7);
    if (to_linear) dst[e] = src[b];
    else dst[b] = src[e];
  }
}
}  // namespace

extern "C" {

int vflip_bricks_to_linear(vflip_ctx* ctx, int nx, int ny, int nz, const float* bricked, float* linear) {
  int rc;
  if ((rc = check_dims(ctx, nx, ny, nz))) return rc;
  if (!bricked || !linear) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  size_t n = (size_t)nx * ny * nz;
  bricks_kernel<<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(bricked, linear, nx, ny, nz, true);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_linear_to_bricks(vflip_ctx* ctx, int nx, int ny, int nz, const float* linear, float* bricked) {
  int rc;
  if ((rc = check_dims(ctx, nx, ny, nz))) return rc;
  if (!bricked || !linear) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  size_t n = (size_t)nx * ny * nz;
  bricks_kernel<<<grid_for(n, 256, ctx->num_sms), 256, 0, ctx->stream>>>(linear, bricked, nx, ny, nz, false);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_emit_tracers(vflip_ctx* ctx, const float* tracers, int n, float h, float lx, float ly, float lz, float cx,
                       float cy, float cz, float r, int count, unsigned seed, float* out, int capacity, int* n_out) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (n < 0 || count < 0 || capacity < 0 || (n > 0 && !tracers) || !out || !n_out || !(h > 0) || !(r >= 0))
    return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  if (n > 0 && out == tracers) return ctx->fail(VFLIP_ERR_ARG, "out aliases the tracers");
  int *keep, *pos;
  VF_ALLOC(keep, int, "tr_keep", (size_t)n + 1);
  VF_ALLOC(pos, int, "tr_pos", (size_t)n + 1);
  const float4* tr = reinterpret_cast<const float4*>(tracers);
  tracer_keep_kernel<<<grid_for((size_t)n + 1, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(tr, n, h, lx, ly, lz,
                                                                                            keep);
  VF_LAUNCH_CHECK();
  int rc;
  if ((rc = exclusive_scan(ctx, keep, pos, (size_t)n + 1))) return rc;
  int m = 0;
  VF_CUDA(cudaMemcpyAsync(&m, pos + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  *n_out = m + count;
  if ((long long)m + count > capacity)
    return ctx->fail(VFLIP_ERR_TOO_LARGE, "%d tracers do not fit a capacity of %d", m + count, capacity);
  float4* o = reinterpret_cast<float4*>(out);
  if (n > 0) {
    tracer_compact_kernel<<<grid_for(n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(tr, n, keep, pos, o);
    VF_LAUNCH_CHECK();
  }
  if (count > 0) {
    tracer_emit_kernel<<<grid_for(count, 128, ctx->num_sms * 8), 128, 0, ctx->stream>>>(o, pos + n, count, seed, r, cx,
                                                                                      cy, cz);
    VF_LAUNCH_CHECK();
  }
  return VFLIP_OK;
}

}  // extern "C"

static int advect_tracers_impl(vflip_ctx* ctx, int ni, int nj, int nk, float h, float* tracers, int n,
                               const float* u, const float* v, const float* w, const float* nodal_phi, float dt,
                               float dens_decay, const vflip_subdomain* sub) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (n < 0 || (n > 0 && !tracers) || !u || !v || !w || !nodal_phi) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  Nest nest;
  if ((rc = make_nest(ctx, sub, &nest))) return rc;
  if (n == 0) return VFLIP_OK;
  const double hd = h, ih = inv_pow2(h);
  GridView gu{u, ni + 1, nj, nk, hd, 0.5, 0.0, 0.0, ih}, gv{v, ni, nj + 1, nk, hd, 0.0, 0.5, 0.0, ih},
      gw{w, ni, nj, nk + 1, hd, 0.0, 0.0, 0.5, ih}, gp{nodal_phi, ni + 1, nj + 1, nk + 1, hd, 0.5, 0.5, 0.5, ih};
  float4* tr = reinterpret_cast<float4*>(tracers);
  const int grid = grid_for(n, 128, ctx->num_sms * 8);
  if (sub)
    advect_tracers_kernel<true><<<grid, 128, 0, ctx->stream>>>(tr, n, gu, gv, gw, gp, dt, dens_decay, nest);
  else
    advect_tracers_kernel<false><<<grid, 128, 0, ctx->stream>>>(tr, n, gu, gv, gw, gp, dt, dens_decay, nest);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

extern "C" {

int vflip_advect_tracers(vflip_ctx* ctx, int ni, int nj, int nk, float h, float* tracers, int n, const float* u,
                         const float* v, const float* w, const float* nodal_phi, float dt, float dens_decay) {
  return advect_tracers_impl(ctx, ni, nj, nk, h, tracers, n, u, v, w, nodal_phi, dt, dens_decay, nullptr);
}

int vflip_advect_tracers_nested(vflip_ctx* ctx, int ni, int nj, int nk, float h, float* tracers, int n,
                                const float* u, const float* v, const float* w, const float* nodal_phi, float dt,
                                float dens_decay, const vflip_subdomain* sub) {
  if (ctx && !sub) return ctx->fail(VFLIP_ERR_ARG, "null subdomain");
  return advect_tracers_impl(ctx, ni, nj, nk, h, tracers, n, u, v, w, nodal_phi, dt, dens_decay, sub);
}

int vflip_emit_tracers_nested(vflip_ctx* ctx, const float* tracers, int n, float h, float lx, float ly, float lz,
                              float cx, float cy, float cz, float r, int count, unsigned seed, int ni, int nj, int nk,
                              const float* nodal_phi, const vflip_subdomain* sub, float* out, int capacity,
                              int* n_out) {
  if (!ctx) return VFLIP_ERR_ARG;
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!sub || !nodal_phi) return ctx->fail(VFLIP_ERR_ARG, "null subdomain or phi");
  Nest nest;
  if ((rc = make_nest(ctx, sub, &nest))) return rc;
  const size_t snc = (size_t)sub->ni * sub->nj * sub->nk;
  if (4.0 * (double)snc > 2147483000.0) return ctx->fail(VFLIP_ERR_TOO_LARGE, "subdomain too large for seeding");
  if ((rc = vflip_emit_tracers(ctx, tracers, n, h, lx, ly, lz, cx, cy, cz, r, count, seed, out, capacity, n_out)))
    return rc;
  const int m = *n_out, ncand = (int)(4 * snc);
  int *flag, *pos;
  VF_ALLOC(flag, int, "ts_flag", (size_t)ncand + 1);
  VF_ALLOC(pos, int, "ts_pos", (size_t)ncand + 1);
  const double hd = h, ih = inv_pow2(h);
  GridView gp{nodal_phi, ni + 1, nj + 1, nk + 1, hd, 0.5, 0.5, 0.5, ih};
  tracer_seed_flag_kernel<<<grid_for((size_t)ncand + 1, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      gp, nest, sub->ni, sub->nj, (uint32_t)seed, ncand, flag);
  VF_LAUNCH_CHECK();
  if ((rc = exclusive_scan(ctx, flag, pos, (size_t)ncand + 1))) return rc;
  int s = 0;
  VF_CUDA(cudaMemcpyAsync(&s, pos + ncand, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  *n_out = m + s;
  if ((long long)m + s > capacity)
    return ctx->fail(VFLIP_ERR_TOO_LARGE, "%d tracers do not fit a capacity of %d", m + s, capacity);
  tracer_seed_write_kernel<<<grid_for(ncand, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      gp, nest, sub->ni, sub->nj, (uint32_t)seed, ncand, flag, pos, m, reinterpret_cast<float4*>(out));
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

int vflip_write_tracers(vflip_ctx* ctx, const float* tracers, int n, float lx, const char* dir, int frame) {
  if (!ctx) return VFLIP_ERR_ARG;
  if (n < 0 || (n > 0 && !tracers) || !dir) return ctx->fail(VFLIP_ERR_ARG, "bad argument");
  std::vector<float> host((size_t)n * 4);
  if (n > 0) {
    float* rec;
    VF_ALLOC(rec, float, "tr_rec", (size_t)n * 4);
    tracer_records_kernel<<<grid_for(n, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
        reinterpret_cast<const float4*>(tracers), n, lx, reinterpret_cast<float4*>(rec));
    VF_LAUNCH_CHECK();
    VF_CUDA(cudaMemcpyAsync(host.data(), rec, sizeof(float) * 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  }
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  char name[4096];
  if (snprintf(name, sizeof name, "%s/Particle_data%04d.bin", dir, frame) >= (int)sizeof name)
    return ctx->fail(VFLIP_ERR_ARG, "path too long");
  FILE* f = fopen(name, "wb");
  if (!f) return ctx->fail(VFLIP_ERR_ARG, "cannot open %s for writing", name);
  const size_t wrote = n > 0 ? fwrite(host.data(), sizeof(float) * 4, (size_t)n, f) : 0;
  const int closed = fclose(f);
  if (wrote != (size_t)n || closed != 0) return ctx->fail(VFLIP_ERR_ARG, "short write to %s", name);
  return VFLIP_OK;
}

}  // extern "C"

extern "C" {

int vflip_plume_sources(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, float* rho, float* temp, float* v,
                        float cx, float cy, float cz, float radius, float dens_value, float heat_value, float alpha,
                        float beta) {
  int rc;
  if ((rc = check_dims(ctx, ni, nj, nk))) return rc;
  if (!rho || !temp || !v) return ctx->fail(VFLIP_ERR_ARG, "null pointer");
  size_t nc = (size_t)ni * nj * nk, nv = (size_t)ni * (nj + 1) * nk;
  plume_sources_kernel<<<grid_for(nc, 256, ctx->num_sms), 256, 0, ctx->stream>>>(rho, temp, ni, nj, nk, h, cx, cy, cz,
                                                                                radius, dens_value, heat_value);
  VF_LAUNCH_CHECK();
  buoyancy_kernel<<<grid_for(nv, 256, ctx->num_sms), 256, 0, ctx->stream>>>(rho, temp, v, ni, nj, nk, dt, alpha, beta);
  VF_LAUNCH_CHECK();
  return VFLIP_OK;
}

}  // extern "C"

extern "C" {

int vflip_set_profiling(vflip_ctx* ctx, int enable) {
  if (!ctx) return VFLIP_ERR_ARG;
  ctx->profiling = enable != 0;
  ctx->prof_used = 0;
  return VFLIP_OK;
}

int vflip_profile_sweeps(vflip_ctx* ctx, int* launches, double* total_ms, double* cells) {
  if (!ctx) return VFLIP_ERR_ARG;
  const double fine = (double)ctx->prof_fine_n;
  int rc = vflip_profile_kernels(ctx, VFLIP_PROF_FINE_SWEEP, launches, total_ms);
  if (cells) *cells = fine;
  if (rc == VFLIP_OK) ctx->prof_used = 0;
  return rc;
}

int vflip_profile_kernels(vflip_ctx* ctx, int kind, int* launches, double* total_ms) {
  if (!ctx) return VFLIP_ERR_ARG;
  VF_CUDA(cudaStreamSynchronize(ctx->stream));
  double tot = 0.0;
  int cnt = 0;
  for (size_t q = 0; q < ctx->prof_used; ++q) {
    if (ctx->prof_events[q].tag != kind) continue;
    float ms = 0.0f;
    VF_CUDA(cudaEventElapsedTime(&ms, ctx->prof_events[q].a, ctx->prof_events[q].b));
    tot += ms;
    ++cnt;
  }
  if (launches) *launches = cnt;
  if (total_ms) *total_ms = tot;
  return VFLIP_OK;
}

unsigned long long vflip_launch_count(const vflip_ctx* ctx) { return ctx ? ctx->launches : 0ull; }

}  // extern "C"

// ============================================================== no-allocation smoother
// vflip_rbgs_noalloc: the red-black smoother of vflip_rbgs for callers that
// must not allocate device memory.  Its ping-pong buffer is the file-scope
// array below; each GPU that loads this library holds it until the process
// exits.  Host code never dereferences the symbol: the device address is
// fetched with cudaGetSymbolAddress once per device, with that device current,
// the first time the entry point runs on it.
namespace {

static __device__ __align__(256) double vflip_noalloc_scratch[VFLIP_NOALLOC_MAX_CELLS];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// Device address of the scratch array and SM count for the current device,
// looked up once per device (the first call should therefore come before any
// stream capture).
cudaError_t noalloc_setup(double** ptr, int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, vflip_noalloc_scratch);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g_noalloc_sms[dev] = n;
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *ptr = g_noalloc_ptr[dev];
  *sms = g_noalloc_sms[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int vflip_rbgs_noalloc(void* stream, int ni, int nj, int nk, const double* diag, const double* xp,
                                  const double* yp, const double* zp, const double* b, double* x, int iterations) {
  if (ni <= 0 || nj <= 0 || nk <= 0 || !diag || !xp || !yp || !zp || !b || !x || iterations < 0)
    return VFLIP_ERR_ARG;
  const size_t n = (size_t)ni * nj * nk;
  if (n > (size_t)VFLIP_NOALLOC_MAX_CELLS) return VFLIP_ERR_TOO_LARGE;
  double* scratch = nullptr;
  int sms = 0;
  if (noalloc_setup(&scratch, &sms) != cudaSuccess) return VFLIP_ERR_CUDA;
  if (iterations == 0) return VFLIP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Dims d{ni, nj, nk};
  SweepShape sh = sweep_shape<double>(d, sms);
  if (sh.smem > 200 * 1024 || sh.grid_y * sh.grid_z > kMaxPartials) return VFLIP_ERR_ARG;
  auto kern = rbgs_sweep_kernel<double, double, false, false, false, kSweepBlock>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
    return VFLIP_ERR_CUDA;
  SweepArgs<double, double> a{};
  a.b = b;
  a.diag = diag;
  a.xp = xp;
  a.yp = yp;
  a.zp = zp;
  a.xc = nullptr;
  a.ni = ni;
  a.nj = nj;
  a.nk = nk;
  a.tyo = sh.tyo;
  a.kz = sh.kz;
  a.plane_stride = sh.plane_stride;
  a.dot_partial = nullptr;
  // ping-pong between x and the scratch array; every sweep writes all cells
  // of its output, so the scratch needs no clearing between calls
  double* cur = x;
  for (int s = 0; s < iterations; ++s) {
    double* out = (cur == x) ? scratch : x;
    a.x_in = cur;
    a.x_out = out;
    kern<<<dim3(sh.grid_y, sh.grid_z), kSweepBlock, sh.smem, st>>>(a);
    if (cudaGetLastError() != cudaSuccess) return VFLIP_ERR_CUDA;
    cur = out;
  }
  if (cur != x && cudaMemcpyAsync(x, cur, sizeof(double) * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return VFLIP_ERR_CUDA;
  return VFLIP_OK;
}
