// Batched MGPCG as ONE persistent cooperative kernel: every system's PCG
// loop (AlgebraicMultigrid.h:189-301) and V(4,4)-cycle (:130-188) for a set
// of independent systems of uneven sizes.
//
// The kernel walks one phase program for the whole batch.  A phase is a work
// list of (system, chunk) items - a chunk is a run of cells (or coarse cells)
// of one level of one system - and the CTAs take items grid-stride; a grid
// barrier separates dependent phases, and every CTA meets every barrier (no
// CTA leaves the program early).  Per PCG iteration:
//   V-cycle: for each level l: four fused red-black sweeps (16 x 8 x 4
//            cell tiles with a two-cell halo, out of place, the first from
//            x = 0: amgPrecond zero-fills x), then b_{l+1} = R (b_l - A_l x_l); the coarsest
//            level of each system (one CTA per system: the FP64
//            band-Cholesky solve, or red-black sweeps in shared memory); up:
//            four sweeps, the first on x + P x_{l+1}; the last sweep of
//            level 0 also forms z.r (rho, beta);
//   s = z + beta s; q = A s with s.q (alpha); x += alpha s, r -= alpha q
//   with |r|_inf (the stop test); systems that converged drop out.
// A sweep tile follows rbgs_sweep_tile_kernel's scheme and every smoother's
// arithmetic, so the V-cycle's values are the single-system kernels' (the
// reductions are grouped per item instead).
//
// Reductions are deterministic: every item writes its partial to a slot of
// its own, and after the barrier one CTA per system folds that system's
// slots in index order.  Vectors written inside the kernel are read through
// L2 (ld.global.cg): another SM's earlier writes are visible after a grid
// barrier, which a per-SM L1 copy would not guarantee.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "pcg_kernels.cuh"

namespace vflip {

constexpr int kBatchThreads = 256;
constexpr int kBatchMaxLevels = 12;

template <typename T>
__device__ __forceinline__ typename Num<T>::Acc ldcg(const T* p) {
  return (typename Num<T>::Acc)__ldcg(p);
}

template <typename S, typename V>
struct BatchLevel {
  int ni, nj, nk;
  const S* diag;
  const S* xp;
  const S* yp;
  const S* zp;
  V* b;  // level rhs (level 0: the PCG residual r)
  V* x;  // level solution (level 0: z); every sweep sequence ends here
  V* t;  // the other buffer of the out-of-place sweeps
  int ntx, nty;  // sweep tiles (kBTX x kBTY x kBTZ cells) along x and y; tile t = tx + ntx (ty + nty tz)
};

template <typename S0, typename SC, typename V>
struct BatchSys {
  int nl;                                  // levels (>= 2)
  BatchLevel<S0, V> fine;
  BatchLevel<SC, V> lv[kBatchMaxLevels];   // lv[l], 1 <= l < nl
  V *x, *s, *q;                            // PCG vectors (r = fine.b, z = fine.x)
  const double* rhs;
  double* result;
  PcgScalars* st;
  int* it;                                 // iterations
  int* state;                              // 1 iterating, 0 converged, 2 stopped on a zero or NaN rho
  // coarsest level: the FP64 band-Cholesky factor (when on and valid), else sweeps
  int direct, bw, sweeps;
  const double* L;
  const double* rinv;
  const int* ok;
  double tol_factor;
};

struct BatchPlan {
  int nsys, lmax, maxit, chunk;
  // items of each level's cell phases and of the restriction into level
  // l+1, as prefix sums over the systems: the items of system s at level l
  // are [cell_pre[l][s], cell_pre[l][s+1]); a system without that level has none
  const int* cell_pre;   // [lmax][nsys+1] (level 0: the PCG vector phases)
  const int* rest_pre;   // [lmax][nsys+1]
  const int* sweep_pre;  // [lmax][nsys+1] sweep tiles of the levels a system smooths
  double* part;         // [nsys][part_stride] reduction slots
  int part_stride;
  int* active;          // [2] systems still iterating, alternating per iteration
  int smem_doubles;     // dynamic shared memory (doubles): the sweeps' plane window, the coarsest phase
};

// the system whose item range holds `item` (pre is non-decreasing)
__device__ __forceinline__ int batch_find(const int* pre, int nsys, int item) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(pre + mid) <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename S0, typename SC, typename V>
__device__ __forceinline__ bool batch_live(const BatchSys<S0, SC, V>& y) {
  return __ldcg(y.state) == 1;
}

// One fused red-black sweep (both colours, out of place) of one kBTX x kBTY
// x kBTZ tile of a level, as rbgs_sweep_tile_kernel does it: x, b and the
// operator over the tile and a two-cell halo are staged at once, the red
// pass runs over the tile and a one-cell ring, the black pass over the tile,
// and the tile is stored (the halo is recomputed by the neighbouring tiles).
// The same values as every other smoother bit for bit.  ZERO: the incoming
// x is 0; PROLONG: it is x_in + P x_c; DOT: returns this thread's part of
// sum(x_out * b).  Vectors written inside the kernel are read through L2.
constexpr int kBTX = 16, kBTY = 8, kBTZ = 4;
constexpr int kBRX = kBTX + 4, kBRY = kBTY + 4, kBRZ = kBTZ + 4, kBRegion = kBRX * kBRY * kBRZ;

template <typename S, typename V, bool ZERO, bool PROLONG, bool DOT>
__device__ double batch_sweep(const BatchLevel<S, V>& L, const V* x_in, V* x_out, const V* xc, int cni, int cnj,
                              int ti, int tj, int tk, typename Num<V>::Acc* sm) {
  using A = typename Num<V>::Acc;
  A *xs = sm, *bs = sm + kBRegion, *ds = sm + 2 * kBRegion, *xps = sm + 3 * kBRegion, *yps = sm + 4 * kBRegion,
    *zps = sm + 5 * kBRegion;
  const int ni = L.ni, nj = L.nj, nk = L.nk;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const int oi = ti * kBTX - 2, oj = tj * kBTY - 2, ok = tk * kBTZ - 2;
  // the staging loads are issued kGrp cells at a time before their
  // shared-memory stores (a few rounds of memory latency, not one per cell;
  // groups keep the registers of this persistent kernel in bounds)
  constexpr int kIt = (kBRegion + kBatchThreads - 1) / kBatchThreads, kGrp = 4;
#pragma unroll 1
  for (int q0 = 0; q0 < kIt; q0 += kGrp) {
    A xv[kGrp], bv[kGrp], dv[kGrp], cxv[kGrp], cyv[kGrp], czv[kGrp];
#pragma unroll
    for (int u = 0; u < kGrp; ++u) {
      const int e = threadIdx.x + (q0 + u) * kBatchThreads;
      const int ri = e % kBRX, rj = (e / kBRX) % kBRY, rk = e / (kBRX * kBRY);
      const int i = oi + ri, j = oj + rj, k = ok + rk;
      A x = A(0), bb = A(0), d = A(0), cx = A(0), cy = A(0), cz = A(0);
      if (q0 + u < kIt && e < kBRegion && i >= 0 && i < ni && j >= 0 && j < nj && k >= 0 && k < nk) {
        const size_t g = (size_t)i + sy * j + sz * k;
        if (!ZERO) {
          x = ldcg(x_in + g);
          if (PROLONG) x = x + ldcg(xc + lin3(i >> 1, j >> 1, k >> 1, cni, cnj));
        }
        bb = ldcg(L.b + g);
        d = A(ldg(L.diag + g));
        cx = A(ldg(L.xp + g));
        cy = A(ldg(L.yp + g));
        cz = A(ldg(L.zp + g));
      }
      xv[u] = x;
      bv[u] = bb;
      dv[u] = d;
      cxv[u] = cx;
      cyv[u] = cy;
      czv[u] = cz;
    }
#pragma unroll
    for (int u = 0; u < kGrp; ++u) {
      const int e = threadIdx.x + (q0 + u) * kBatchThreads;
      if (q0 + u < kIt && e < kBRegion) {
        xs[e] = xv[u];
        bs[e] = bv[u];
        ds[e] = dv[u];
        xps[e] = cxv[u];
        yps[e] = cyv[u];
        zps[e] = czv[u];
      }
    }
  }
  __syncthreads();
  constexpr int SY = kBRX, SZ = kBRX * kBRY;
  auto pass = [&](int lo, int hx, int hy, int hz, int parity) {
    const int wx = hx - lo, wy = hy - lo, cnt = wx * wy * (hz - lo);
    for (int q = threadIdx.x; q < cnt; q += kBatchThreads) {
      const int ri = lo + q % wx, rj = lo + (q / wx) % wy, rk = lo + q / (wx * wy);
      const int i = oi + ri, j = oj + rj, k = ok + rk;
      if (i < 0 || i >= ni || j < 0 || j >= nj || k < 0 || k >= nk) continue;
      if (((i + j + k) & 1) != parity) continue;
      const int e = ri + SY * rj + SZ * rk;
      A sum = A(0);
      if (k > 0) sum = gs_madd(sum, zps[e - SZ], xs[e - SZ]);
      if (j > 0) sum = gs_madd(sum, yps[e - SY], xs[e - SY]);
      if (i > 0) sum = gs_madd(sum, xps[e - 1], xs[e - 1]);
      if (i < ni - 1) sum = gs_madd(sum, xps[e], xs[e + 1]);
      if (j < nj - 1) sum = gs_madd(sum, yps[e], xs[e + SY]);
      if (k < nk - 1) sum = gs_madd(sum, zps[e], xs[e + SZ]);
      const A d = ds[e];
      xs[e] = (d != A(0)) ? gs_div(bs[e] - sum, d) : A(0);
    }
  };
  pass(1, kBRX - 1, kBRY - 1, kBRZ - 1, 1);  // red: the tile and a one-cell ring
  __syncthreads();
  pass(2, kBRX - 2, kBRY - 2, kBRZ - 2, 0);  // black: the tile
  __syncthreads();
  double dot = 0.0;
  constexpr int cnt = kBTX * kBTY * kBTZ;
  for (int q = threadIdx.x; q < cnt; q += kBatchThreads) {
    const int ri = 2 + q % kBTX, rj = 2 + (q / kBTX) % kBTY, rk = 2 + q / (kBTX * kBTY);
    const int i = oi + ri, j = oj + rj, k = ok + rk;
    if (i >= ni || j >= nj || k >= nk) continue;
    const int e = ri + SY * rj + SZ * rk;
    const V o = cvt<V>(xs[e]);
    x_out[(size_t)i + sy * j + sz * k] = o;
    if (DOT) dot += (double)ldv(&o) * (double)bs[e];
  }
  __syncthreads();  // the next tile restages the region
  return dot;
}

// b_c = R (b - A x) over the coarse cells [c0, c1) (residual_restrict_kernel's arithmetic)
template <typename S, typename V, typename SN>
__device__ __forceinline__ void batch_restrict(const BatchLevel<S, V>& F, const BatchLevel<SN, V>& Cl, size_t c0,
                                               size_t c1) {
  using A = typename Num<V>::Acc;
  const int ni = F.ni, nj = F.nj, nk = F.nk;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  for (size_t e = c0 + threadIdx.x; e < c1; e += kBatchThreads) {
    int I, J, K;
    decode3(e, Cl.ni, Cl.nj, I, J, K);
    A s = A(0);
#pragma unroll
    for (int kk = 0; kk <= 1; ++kk)
#pragma unroll
      for (int jj = 0; jj <= 1; ++jj)
#pragma unroll
        for (int ii = 0; ii <= 1; ++ii) {
          const int i = 2 * I + ii, j = 2 * J + jj, k = 2 * K + kk;
          if (i >= ni || j >= nj || k >= nk) continue;
          const size_t g = lin3(i, j, k, ni, nj);
          A r = ldcg(F.b + g);
          if (k > 0) r = r - A(ldg(F.zp + g - sz)) * ldcg(F.x + g - sz);
          if (j > 0) r = r - A(ldg(F.yp + g - sy)) * ldcg(F.x + g - sy);
          if (i > 0) r = r - A(ldg(F.xp + g - 1)) * ldcg(F.x + g - 1);
          r = r - A(ldg(F.diag + g)) * ldcg(F.x + g);
          if (i < ni - 1) r = r - A(ldg(F.xp + g)) * ldcg(F.x + g + 1);
          if (j < nj - 1) r = r - A(ldg(F.yp + g)) * ldcg(F.x + g + sy);
          if (k < nk - 1) r = r - A(ldg(F.zp + g)) * ldcg(F.x + g + sz);
          s = s + A(0.125) * r;
        }
    Cl.b[e] = cvt<V>(s);
  }
}

// The coarsest level of one system, by one CTA: the FP64 band-Cholesky
// solve (coarse_chol_solve_kernel's steps, its factor read from global
// memory) when the factor is valid, else `sweeps` red-black sweeps from
// zero, staged in shared memory when the level fits.
template <typename SC, typename V>
__device__ void batch_coarsest(const BatchLevel<SC, V>& L, int direct, int bw, const double* Lc, const double* rinv,
                               const int* ok, int sweeps, double* sm, int smem_doubles) {
  using A = typename Num<V>::Acc;
  const int n = L.ni * L.nj * L.nk;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr unsigned FULL = 0xffffffffu;
  if (direct && n <= smem_doubles && __ldg(ok) != 0) {
    double* y = sm;
    const int B1 = bw + 1;
    for (int e = tid; e < n; e += kBatchThreads) y[e] = (double)ldcg(L.b + e);
    __syncthreads();
    for (int kb = 0; kb < n; kb += 32) {
      const int nb = min(32, n - kb);
      if (warp == 0) {
        double yr = lane < nb ? y[kb + lane] : 0.0;
        for (int c = 0; c < nb; ++c) {
          const double lrc =
              (lane > c && lane < nb && lane - c <= bw) ? __ldg(Lc + (size_t)(kb + c) * B1 + (lane - c)) : 0.0;
          const double yc = __shfl_sync(FULL, yr, c) * __ldg(rinv + kb + c);
          if (lane == c) yr = yc;
          else if (lane > c) yr -= lrc * yc;
        }
        if (lane < nb) y[kb + lane] = yr;
      }
      __syncthreads();
      const int r0 = kb + nb, r1 = min(n, kb + nb + bw);
      for (int i = r0 + tid; i < r1; i += kBatchThreads) {
        double s = y[i];
        for (int c = 0; c < nb; ++c) {
          const int d = i - (kb + c);
          if (d <= bw) s -= __ldg(Lc + (size_t)(kb + c) * B1 + d) * y[kb + c];
        }
        y[i] = s;
      }
      __syncthreads();
    }
    const int last = ((n - 1) / 32) * 32;
    for (int kb = last; kb >= 0; kb -= 32) {
      const int nb = min(32, n - kb);
      {
        const int r = tid >> 3, part = tid & 7;
        double s = 0.0;
        if (r < nb) {
          const int c = kb + r;
          for (int d = kb + nb - c + part; d <= bw && c + d < n; d += 8)
            s += __ldg(Lc + (size_t)c * B1 + d) * y[c + d];
        }
        s += __shfl_down_sync(FULL, s, 4, 8);
        s += __shfl_down_sync(FULL, s, 2, 8);
        s += __shfl_down_sync(FULL, s, 1, 8);
        __syncthreads();
        if (r < nb && part == 0) y[kb + r] -= s;
      }
      __syncthreads();
      if (warp == 0) {
        double yr = lane < nb ? y[kb + lane] : 0.0;
        for (int c = nb - 1; c >= 0; --c) {
          const double lcr = (lane < c && c - lane <= bw) ? __ldg(Lc + (size_t)(kb + lane) * B1 + (c - lane)) : 0.0;
          const double xc = __shfl_sync(FULL, yr, c) * __ldg(rinv + kb + c);
          if (lane == c) yr = xc;
          else if (lane < c) yr -= lcr * xc;
        }
        if (lane < nb) y[kb + lane] = yr;
      }
      __syncthreads();
    }
    for (int e = tid; e < n; e += kBatchThreads) L.x[e] = cvt<V>((A)y[e]);
    __syncthreads();
    return;
  }
  const bool staged = (size_t)2 * n * sizeof(A) <= (size_t)smem_doubles * sizeof(double);
  A* xs = reinterpret_cast<A*>(sm);
  A* bs = xs + n;
  const int ni = L.ni, nj = L.nj, nk = L.nk, sy = ni, sz = ni * nj;
  for (int e = tid; e < n; e += kBatchThreads) {
    if (staged) {
      xs[e] = A(0);
      bs[e] = ldcg(L.b + e);
    } else {
      L.x[e] = cvt<V>(A(0));
    }
  }
  if (!staged) __threadfence();
  __syncthreads();
  for (int it = 0; it < sweeps; ++it) {
    for (int parity = 1; parity >= 0; --parity) {
      for (int e = tid; e < n; e += kBatchThreads) {
        const int i = e % ni, j = (e / ni) % nj, k = e / sz;
        if (((i + j + k) & 1) != parity) continue;
        auto X = [&](int q) -> A { return staged ? xs[q] : ldcg(L.x + q); };
        A sum = A(0);
        if (k > 0) sum = gs_madd(sum, A(ldg(L.zp + e - sz)), X(e - sz));
        if (j > 0) sum = gs_madd(sum, A(ldg(L.yp + e - sy)), X(e - sy));
        if (i > 0) sum = gs_madd(sum, A(ldg(L.xp + e - 1)), X(e - 1));
        if (i < ni - 1) sum = gs_madd(sum, A(ldg(L.xp + e)), X(e + 1));
        if (j < nj - 1) sum = gs_madd(sum, A(ldg(L.yp + e)), X(e + sy));
        if (k < nk - 1) sum = gs_madd(sum, A(ldg(L.zp + e)), X(e + sz));
        const A d = A(ldg(L.diag + e));
        const A bb = staged ? bs[e] : ldcg(L.b + e);
        const A v = (d != A(0)) ? gs_div(bb - sum, d) : A(0);
        if (staged) xs[e] = v;
        else L.x[e] = cvt<V>(v);
      }
      if (!staged) __threadfence();  // the next colour reads these values through L2
      __syncthreads();
    }
  }
  if (staged)
    for (int e = tid; e < n; e += kBatchThreads) L.x[e] = cvt<V>(xs[e]);
  __syncthreads();
}

// block sum / max of one double per thread, valid in thread 0 (warp trees, then warps in order)
__device__ __forceinline__ double batch_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kBatchThreads / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

__device__ __forceinline__ double batch_block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kBatchThreads / 32; ++w) s = fmax(s, red[w]);
  __syncthreads();
  return s;
}

enum BatchFold { kFoldInit = 0, kFoldRho = 1, kFoldSZ = 2, kFoldRes = 3 };

template <typename S0, typename SC, typename V>
__global__ void __launch_bounds__(kBatchThreads) batch_pcg_kernel(const BatchSys<S0, SC, V>* __restrict__ sys,
                                                                  const BatchPlan p) {
  namespace cg = cooperative_groups;
  using A = typename Num<V>::Acc;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) double bsm[];
  __shared__ double red[kBatchThreads / 32];
  const int G = gridDim.x, B = blockIdx.x, nsys = p.nsys, CH = p.chunk;

  // every item of level l's cell phase: fn(system, its index, item index
  // within the system, first cell), live systems only (uniform per CTA)
  auto cells = [&](int l, auto&& fn) {
    const int* pre = p.cell_pre + (size_t)l * (nsys + 1);
    const int total = __ldg(pre + nsys);
    for (int item = B; item < total; item += G) {
      const int s = batch_find(pre, nsys, item);
      const BatchSys<S0, SC, V>& y = sys[s];
      if (!batch_live(y)) continue;
      const int local = item - __ldg(pre + s);
      fn(y, s, local, (size_t)local * CH);
    }
  };
  // every sweep tile of level l of the systems that smooth there (live ones):
  // fn(system, its index, tile index within the system, tile x, y, z)
  auto tiles = [&](int l, auto&& fn) {
    const int* pre = p.sweep_pre + (size_t)l * (nsys + 1);
    const int total = __ldg(pre + nsys);
    for (int item = B; item < total; item += G) {
      const int s = batch_find(pre, nsys, item);
      const BatchSys<S0, SC, V>& y = sys[s];
      if (!batch_live(y)) continue;
      const int local = item - __ldg(pre + s);
      const int ntx = l == 0 ? y.fine.ntx : y.lv[l].ntx, nty = l == 0 ? y.fine.nty : y.lv[l].nty;
      fn(y, s, local, local % ntx, (local / ntx) % nty, local / (ntx * nty));
    }
  };
  A* xs = reinterpret_cast<A*>(bsm);  // the sweeps' plane window
  auto slot = [&](int s, int local) -> double* { return p.part + (size_t)s * p.part_stride + local; };
  // one CTA per system folds that system's level-0 slots in index order
  auto fold = [&](int kind) {
    for (int s = B; s < nsys; s += G) {
      const BatchSys<S0, SC, V>& y = sys[s];
      if (kind != kFoldInit && !batch_live(y)) continue;
      const int* cpre = kind == kFoldRho ? p.sweep_pre : p.cell_pre;
      const int cnt = __ldg(cpre + s + 1) - __ldg(cpre + s);
      const bool mx = kind == kFoldInit || kind == kFoldRes;
      double v = 0.0;
      for (int q = threadIdx.x; q < cnt; q += kBatchThreads) {
        const double w = __ldcg(slot(s, q));
        v = mx ? fmax(v, w) : v + w;
      }
      const double tot = mx ? batch_block_max(v, red) : batch_block_sum(v, red);
      if (threadIdx.x == 0) {
        PcgScalars* st = y.st;
        if (kind == kFoldInit) {  // AlgebraicMultigrid.h:211-215
          st->res = tot;
          st->rhs_norm = tot;
          st->tol = y.tol_factor * tot;
          st->converged = tot == 0.0 ? 1 : 0;
          st->rho = 1.0;
          st->beta = 0.0;
          st->bad_rho = 0;
          *y.it = 0;
          *y.state = tot == 0.0 ? 0 : 1;
        } else if (kind == kFoldRho) {
          st->beta = tot / __ldcg(&st->rho);
          st->rho = tot;
          // AlgebraicMultigrid.h:236-252: a zero or NaN rho of the first V-cycle ends the solve
          if (__ldcg(y.it) == 0 && (tot == 0.0 || tot != tot)) {
            st->bad_rho = 1;
            *y.state = 2;
          }
        } else if (kind == kFoldSZ) {
          st->sz = tot;
          st->alpha = __ldcg(&st->rho) / tot;
        } else {
          st->res = tot;
          const int conv = tot <= __ldcg(&st->tol) ? 1 : 0;
          st->converged = conv;
          *y.it = __ldcg(y.it) + 1;
          if (conv) *y.state = 0;
        }
      }
      __syncthreads();
    }
  };

  // ---- r = rhs, x = s = 0, |rhs|_inf (every system: none has a state yet)
  {
    const int total = __ldg(p.cell_pre + nsys);
    for (int item = B; item < total; item += G) {
      const int s = batch_find(p.cell_pre, nsys, item);
      const BatchSys<S0, SC, V>& y = sys[s];
      const int local = item - __ldg(p.cell_pre + s);
      const size_t n = (size_t)y.fine.ni * y.fine.nj * y.fine.nk, c0 = (size_t)local * CH, c1 = min(c0 + CH, n);
      double m = 0.0;
      for (size_t g = c0 + threadIdx.x; g < c1; g += kBatchThreads) {
        const double v = y.rhs[g];
        y.fine.b[g] = cvt<V>((A)v);
        y.x[g] = cvt<V>(A(0));
        y.s[g] = cvt<V>(A(0));
        m = fmax(m, fabs(v));
      }
      const double bm = batch_block_max(m, red);
      if (threadIdx.x == 0) *slot(s, local) = bm;
    }
  }
  if (B == 0 && threadIdx.x == 0) {
    p.active[0] = nsys;  // the first round runs; systems with a zero rhs skip its phases
    p.active[1] = 0;
  }
  grid.sync();
  fold(kFoldInit);
  grid.sync();

  for (int iter = 0; iter < p.maxit; ++iter) {
    if (__ldcg(p.active + (iter & 1)) == 0) break;  // every CTA reads the same count after the barrier
    // ---- V-cycle, down: four sweeps from x = 0 ending in x (t, x, t, x)
    for (int l = 0; l + 1 < p.lmax; ++l) {
      for (int sw = 0; sw < 4; ++sw) {
        tiles(l, [&](const BatchSys<S0, SC, V>& y, int, int, int ti, int tj, int tk) {
          if (l == 0) {
            const BatchLevel<S0, V>& L = y.fine;
            if (sw == 0) batch_sweep<S0, V, true, false, false>(L, nullptr, L.t, nullptr, 0, 0, ti, tj, tk, xs);
            else batch_sweep<S0, V, false, false, false>(L, sw & 1 ? L.t : L.x, sw & 1 ? L.x : L.t, nullptr, 0, 0,
                                                         ti, tj, tk, xs);
          } else {
            const BatchLevel<SC, V>& L = y.lv[l];
            if (sw == 0) batch_sweep<SC, V, true, false, false>(L, nullptr, L.t, nullptr, 0, 0, ti, tj, tk, xs);
            else batch_sweep<SC, V, false, false, false>(L, sw & 1 ? L.t : L.x, sw & 1 ? L.x : L.t, nullptr, 0, 0,
                                                         ti, tj, tk, xs);
          }
        });
        grid.sync();
      }
      {
        const int* pre = p.rest_pre + (size_t)l * (nsys + 1);
        const int total = __ldg(pre + nsys);
        for (int item = B; item < total; item += G) {
          const int s = batch_find(pre, nsys, item);
          const BatchSys<S0, SC, V>& y = sys[s];
          if (!batch_live(y)) continue;
          const size_t c0 = (size_t)(item - __ldg(pre + s)) * CH;
          const BatchLevel<SC, V>& C = y.lv[l + 1];
          const size_t c1 = min(c0 + CH, (size_t)C.ni * C.nj * C.nk);
          if (l == 0) batch_restrict<S0, V, SC>(y.fine, C, c0, c1);
          else batch_restrict<SC, V, SC>(y.lv[l], C, c0, c1);
        }
      }
      grid.sync();
    }
    // ---- the coarsest level of every live system, one CTA each
    for (int s = B; s < nsys; s += G) {
      const BatchSys<S0, SC, V>& y = sys[s];
      if (!batch_live(y)) continue;
      batch_coarsest<SC, V>(y.lv[y.nl - 1], y.direct, y.bw, y.L, y.rinv, y.ok, y.sweeps, bsm, p.smem_doubles);
    }
    grid.sync();
    // ---- V-cycle, up: x + P x_c, then four sweeps ending in x; the last
    // sweep of level 0 forms the partial z.r
    for (int l = p.lmax - 2; l >= 0; --l) {
      for (int sw = 0; sw < 4; ++sw) {
        const bool last = l == 0 && sw == 3;
        tiles(l, [&](const BatchSys<S0, SC, V>& y, int s, int local, int ti, int tj, int tk) {
          const BatchLevel<SC, V>& C = y.lv[l + 1];
          if (l == 0) {
            const BatchLevel<S0, V>& L = y.fine;
            double d = 0.0;
            if (sw == 0) batch_sweep<S0, V, false, true, false>(L, L.x, L.t, C.x, C.ni, C.nj, ti, tj, tk, xs);
            else if (last) d = batch_sweep<S0, V, false, false, true>(L, L.t, L.x, nullptr, 0, 0, ti, tj, tk, xs);
            else batch_sweep<S0, V, false, false, false>(L, sw & 1 ? L.t : L.x, sw & 1 ? L.x : L.t, nullptr, 0, 0,
                                                         ti, tj, tk, xs);
            if (last) {
              const double bs = batch_block_sum(d, red);
              if (threadIdx.x == 0) *slot(s, local) = bs;
            }
          } else {
            const BatchLevel<SC, V>& L = y.lv[l];
            if (sw == 0) batch_sweep<SC, V, false, true, false>(L, L.x, L.t, C.x, C.ni, C.nj, ti, tj, tk, xs);
            else batch_sweep<SC, V, false, false, false>(L, sw & 1 ? L.t : L.x, sw & 1 ? L.x : L.t, nullptr, 0, 0,
                                                         ti, tj, tk, xs);
          }
        });
        grid.sync();
      }
    }
    fold(kFoldRho);
    grid.sync();
    // ---- s = z + beta s
    cells(0, [&](const BatchSys<S0, SC, V>& y, int, int, size_t c0) {
      const size_t c1 = min(c0 + CH, (size_t)y.fine.ni * y.fine.nj * y.fine.nk);
      const double beta = __ldcg(&y.st->beta);
      for (size_t g = c0 + threadIdx.x; g < c1; g += kBatchThreads)
        y.s[g] = cvt<V>((A)((double)ldcg(y.fine.x + g) + beta * (double)ldcg(y.s + g)));
    });
    grid.sync();
    // ---- q = A s, s.q (pcg_spmv_dot_kernel's arithmetic)
    cells(0, [&](const BatchSys<S0, SC, V>& y, int s, int local, size_t c0) {
      const BatchLevel<S0, V>& F = y.fine;
      const int ni = F.ni, nj = F.nj, nk = F.nk;
      const size_t sy = (size_t)ni, sz = (size_t)ni * nj, c1 = min(c0 + CH, (size_t)ni * nj * nk);
      double dot = 0.0;
      for (size_t g = c0 + threadIdx.x; g < c1; g += kBatchThreads) {
        int i, j, k;
        decode3(g, ni, nj, i, j, k);
        const A sc = ldcg(y.s + g);
        A acc = A(0);
        if (k > 0) acc = acc + ldg(F.zp + g - sz) * ldcg(y.s + g - sz);
        if (j > 0) acc = acc + ldg(F.yp + g - sy) * ldcg(y.s + g - sy);
        if (i > 0) acc = acc + ldg(F.xp + g - 1) * ldcg(y.s + g - 1);
        acc = acc + ldg(F.diag + g) * sc;
        if (i < ni - 1) acc = acc + ldg(F.xp + g) * ldcg(y.s + g + 1);
        if (j < nj - 1) acc = acc + ldg(F.yp + g) * ldcg(y.s + g + sy);
        if (k < nk - 1) acc = acc + ldg(F.zp + g) * ldcg(y.s + g + sz);
        const V qq = cvt<V>(acc);
        y.q[g] = qq;
        dot += (double)sc * (double)ldv(&qq);
      }
      const double bs = batch_block_sum(dot, red);
      if (threadIdx.x == 0) *slot(s, local) = bs;
    });
    grid.sync();
    fold(kFoldSZ);
    grid.sync();
    // ---- x += alpha s, r -= alpha q, |r|_inf (pcg_update_kernel's arithmetic)
    cells(0, [&](const BatchSys<S0, SC, V>& y, int s, int local, size_t c0) {
      const size_t c1 = min(c0 + CH, (size_t)y.fine.ni * y.fine.nj * y.fine.nk);
      const double alpha = __ldcg(&y.st->alpha), nalpha = -alpha;
      double m = 0.0;
      for (size_t g = c0 + threadIdx.x; g < c1; g += kBatchThreads) {
        const double xv = (double)ldcg(y.x + g) + alpha * (double)ldcg(y.s + g);
        const double rv = (double)ldcg(y.fine.b + g) + nalpha * (double)ldcg(y.q + g);
        const V rt = cvt<V>((A)rv);
        y.x[g] = cvt<V>((A)xv);
        y.fine.b[g] = rt;
        m = fmax(m, fabs((double)ldv(&rt)));
      }
      const double bm = batch_block_max(m, red);
      if (threadIdx.x == 0) *slot(s, local) = bm;
    });
    if (B == 0 && threadIdx.x == 0) p.active[(iter + 1) & 1] = 0;
    grid.sync();
    // the stop test; count the systems still iterating for the next round
    fold(kFoldRes);
    {
      int live = 0;
      if (threadIdx.x == 0)
        for (int s = B; s < nsys; s += G) live += __ldcg(sys[s].state) == 1 ? 1 : 0;
      if (threadIdx.x == 0 && live) atomicAdd(p.active + ((iter + 1) & 1), live);
    }
    grid.sync();
  }
  // ---- results (x to FP64)
  for (int s = 0; s < nsys; ++s) {
    const BatchSys<S0, SC, V>& y = sys[s];
    const size_t n = (size_t)y.fine.ni * y.fine.nj * y.fine.nk;
    for (size_t g = (size_t)B * kBatchThreads + threadIdx.x; g < n; g += (size_t)G * kBatchThreads)
      y.result[g] = (double)ldcg(y.x + g);
  }
}

}  // namespace vflip
