// The learned preconditioner's U-Net: parameters, activation buffers, the
// forward / backward schedules over the tensor-core convolutions, Adam, and
// the C ABI (vflip_unet_*).  No reference counterpart: the reference solves
// with plain MGPCG only.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>

#include "../../include/vflip.h"
#include "unet_kernels.cuh"
#include "unet_net.h"

namespace vflip {
namespace unet {

const LayerSpec kSpec[kNumLayers] = {
    {16, 16, 1},  {16, 16, 1}, {16, 32, 1}, {32, 32, 1}, {32, 64, 1}, {64, 64, 1}, {64, 128, 1}, {128, 128, 1},
    {192, 64, 1}, {64, 64, 1}, {96, 32, 1}, {32, 32, 1}, {48, 16, 1}, {16, 16, 1}, {16, 16, 0},
};

namespace {

constexpr size_t kConvSmemMax = 200 * 1024;
constexpr size_t kConvSmemFloor = 100 * 1024;   // at most two CTAs (2 x <= 256 TMEM columns) per SM
constexpr size_t kWgradSmemMax = 200 * 1024;
constexpr size_t kWgradSmemFloor = 116 * 1024;  // one CTA (512 TMEM columns) per SM

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 4-D map over a channels-last BF16 view: dims (c, X, Y, Z), box (8, bx, by, bz)
bool make_map(CUtensorMap* m, const View& v, int X, int Y, int Z, int bx, int by, int bz) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)v.c, (cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
  const cuuint64_t row = (cuuint64_t)v.ctot * 2;
  const cuuint64_t strides[3] = {row, row * X, row * X * Y};
  const cuuint32_t box[4] = {8, (cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)(v.p + v.coff), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

uint32_t pow2_cols(int n) {
  uint32_t c = 32;
  while ((int)c < n) c <<= 1;
  return c;
}

int grid1(size_t n, int sms) {
  size_t g = (n + 255) / 256;
  return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)sms * 8));
}

bool view_ok(const View& v) {
  return v.p && v.c > 0 && v.c % 8 == 0 && v.coff % 8 == 0 && v.ctot % 8 == 0 && v.coff + v.c <= v.ctot &&
         (reinterpret_cast<uintptr_t>(v.p) & 15) == 0;
}

}  // namespace

int Net::fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  err = buf;
  return code;
}

#define NET_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return fail(VFLIP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)
#define NET_LAUNCH()                                                                         \
  do {                                                                                       \
    ++launches;                                                                              \
    cudaError_t e_ = cudaGetLastError();                                                     \
    if (e_ != cudaSuccess) return fail(VFLIP_ERR_CUDA, "launch: %s", cudaGetErrorString(e_)); \
  } while (0)
#define NET_TRY(expr)         \
  do {                        \
    int rc_ = (expr);         \
    if (rc_) return rc_;      \
  } while (0)

struct Net::Acts {
  int X[4] = {}, Y[4] = {}, Z[4] = {};
  size_t V[4] = {};
  __nv_bfloat16 *in0, *a_e0a, *cat0, *p1, *a_e1a, *cat1, *p2, *a_e2a, *cat2, *p3, *a_b1, *b3, *a_d2a, *d2, *a_d1a,
      *d1, *a_d0a, *d0;
  __nv_bfloat16 *g_out, *g_d0, *g_d0a, *g_cat0, *g_d1, *g_d1a, *g_cat1, *g_d2, *g_d2a, *g_cat2, *g_b3, *g_b1, *g_p3,
      *g_e2a, *g_p2, *g_e1a, *g_p1, *g_e0a;
  float* out2 = nullptr;  // FP32 output of the last forward (kept for the loss)
  bool have_forward = false;
};

Net::Net(int dev, cudaStream_t s, unsigned long long seed) : device(dev), stream(s) {
  if (cudaSetDevice(device) != cudaSuccess) {
    init_rc = fail(VFLIP_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    return;
  }
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
  size_t off = 0;
  for (int l = 0; l < kNumLayers; ++l) {
    woff[l] = off;
    off += (size_t)kSpec[l].cout * kSpec[l].cin * 27;
    boff[l] = off;
    off += (size_t)kSpec[l].cout;
  }
  nparams = (int)off;
  // He-normal initialisation (seeded), zero biases; OUT keeps only its first 2 output rows
  std::vector<float> h(nparams, 0.0f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kNumLayers; ++l) {
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)(kSpec[l].cin * 27)));
    const int rows = l == OUT ? kOutValid : kSpec[l].cout;
    for (int co = 0; co < rows; ++co)
      for (int k = 0; k < kSpec[l].cin * 27; ++k) h[woff[l] + (size_t)co * kSpec[l].cin * 27 + k] = nd(rng);
  }
  const size_t pb = sizeof(float) * (size_t)nparams;
  size_t packed = 0;
  for (int l = 0; l < kNumLayers; ++l) packed += (size_t)27 * kSpec[l].cin * kSpec[l].cout;
  void* wmem = nullptr;
  if (cudaMalloc(&params, pb) != cudaSuccess || cudaMalloc(&grads, pb) != cudaSuccess ||
      cudaMalloc(&adam_m, pb) != cudaSuccess || cudaMalloc(&adam_v, pb) != cudaSuccess ||
      cudaMalloc(&wmem, 2 * packed * sizeof(__nv_bfloat16)) != cudaSuccess ||
      cudaMalloc(&d_error, sizeof(int)) != cudaSuccess) {
    init_rc = fail(VFLIP_ERR_NOMEM, "cudaMalloc failed for the network parameters");
    return;
  }
  __nv_bfloat16* w = static_cast<__nv_bfloat16*>(wmem);
  for (int l = 0; l < kNumLayers; ++l) {
    const size_t n = (size_t)27 * kSpec[l].cin * kSpec[l].cout;
    wf[l] = w;
    wd[l] = w + packed;
    w += n;
  }
  if (cudaMemsetAsync(adam_m, 0, pb, stream) != cudaSuccess || cudaMemsetAsync(adam_v, 0, pb, stream) != cudaSuccess ||
      cudaMemsetAsync(grads, 0, pb, stream) != cudaSuccess || cudaMemsetAsync(d_error, 0, sizeof(int), stream) != cudaSuccess ||
      cudaMemcpyAsync(params, h.data(), pb, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    init_rc = fail(VFLIP_ERR_CUDA, "parameter upload failed");
    return;
  }
  if (!encode_fn()) {
    init_rc = fail(VFLIP_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    return;
  }
  if (cudaFuncSetAttribute(conv3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kConvSmemMax) !=
          cudaSuccess ||
      cudaFuncSetAttribute(conv3_wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWgradSmemMax) !=
          cudaSuccess) {
    init_rc = fail(VFLIP_ERR_CUDA, "cannot raise the dynamic shared memory limit");
    return;
  }
  init_rc = repack();
}

Net::~Net() {
  cudaSetDevice(device);
  cudaFree(params);
  cudaFree(grads);
  cudaFree(adam_m);
  cudaFree(adam_v);
  cudaFree(wf[0]);
  cudaFree(d_error);
  cudaFree(act_mem);
  for (auto& s : scratch_) cudaFree(s.first);
  if (fwd_exec) cudaGraphExecDestroy(fwd_exec);
  if (fwd_graph) cudaGraphDestroy(fwd_graph);
  if (cap_stream) cudaStreamDestroy(cap_stream);
  delete acts;
}

void* Net::scratch(size_t bytes, int slot) {
  if ((int)scratch_.size() <= slot) scratch_.resize(slot + 1, {nullptr, 0});
  auto& s = scratch_[slot];
  if (s.second >= bytes) return s.first;
  cudaFree(s.first);
  s = {nullptr, 0};
  if (cudaMalloc(&s.first, bytes) != cudaSuccess) return nullptr;
  s.second = bytes;
  return s.first;
}

int Net::pack(const float* w, __nv_bfloat16* out, int cin, int cout, int flip) {
  const size_t n = (size_t)27 * cin * cout;
  pack_weights_kernel<<<grid1(n, num_sms), 256, 0, stream>>>(w, out, cin, cout, flip);
  NET_LAUNCH();
  return VFLIP_OK;
}

int Net::repack() {
  for (int l = 0; l < kNumLayers; ++l) {
    NET_TRY(pack(params + woff[l], wf[l], kSpec[l].cin, kSpec[l].cout, 0));
    NET_TRY(pack(params + woff[l], wd[l], kSpec[l].cin, kSpec[l].cout, 1));
  }
  return VFLIP_OK;
}

int Net::get_params(float* host) const {
  if (cudaMemcpyAsync(host, params, sizeof(float) * nparams, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return VFLIP_ERR_CUDA;
  return VFLIP_OK;
}

int Net::set_params(const float* host) {
  NET_CUDA(cudaMemcpyAsync(params, host, sizeof(float) * nparams, cudaMemcpyHostToDevice, stream));
  NET_CUDA(cudaMemsetAsync(adam_m, 0, sizeof(float) * nparams, stream));
  NET_CUDA(cudaMemsetAsync(adam_v, 0, sizeof(float) * nparams, stream));
  adam_t = 0;
  NET_TRY(repack());
  NET_CUDA(cudaStreamSynchronize(stream));
  return VFLIP_OK;
}

int Net::copy_grads(float* dst) const {
  if (cudaMemcpyAsync(dst, grads, sizeof(float) * nparams, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    return VFLIP_ERR_CUDA;
  return VFLIP_OK;
}

int Net::sync_error() {
  int h = 0;
  NET_CUDA(cudaMemcpyAsync(&h, d_error, sizeof(int), cudaMemcpyDeviceToHost, stream));
  NET_CUDA(cudaStreamSynchronize(stream));
  if (h) {
    cudaMemsetAsync(d_error, 0, sizeof(int), stream);
    return fail(VFLIP_ERR_CUDA, "convolution copy pipeline timed out");
  }
  return VFLIP_OK;
}

// ---------------------------------------------------------------- single ops
int Net::conv(const View& in, int X, int Y, int Z, const __nv_bfloat16* wpacked, const float* bias, int cin, int cout,
              int relu, const View* mask, const View* out, float* outf, int ofstride, int ofvalid) {
  if (X <= 0 || Y <= 0 || Z <= 0) return fail(VFLIP_ERR_ARG, "conv: empty grid");
  if (cin % 16 || cout % 16 || cout > 256 || cin < 16) return fail(VFLIP_ERR_ARG, "conv: channels %d -> %d", cin, cout);
  if (!view_ok(in) || in.c != cin) return fail(VFLIP_ERR_ARG, "conv: bad input view");
  if (out && (!view_ok(*out) || out->c != cout)) return fail(VFLIP_ERR_ARG, "conv: bad output view");
  if (mask && (!view_ok(*mask) || mask->c != cout)) return fail(VFLIP_ERR_ARG, "conv: bad mask view");
  if (!out && !outf) return fail(VFLIP_ERR_ARG, "conv: no output");
  if (outf && (ofvalid < 0 || ofvalid > cout || ofstride < ofvalid)) return fail(VFLIP_ERR_ARG, "conv: bad fp32 output");
  // weights resident when every tap fits beside the two slabs; else the
  // widest channel group whose slabs leave room for a ring of >= 8 slots
  const int nch = cin / 8;
  int cc = 0, ring = 0;
  const size_t full = 2 * (size_t)nch * kPlane + (size_t)27 * nch * cout * 16;
  if (full <= kConvSmemMax) {
    cc = nch;
    ring = 27;
  } else {
    for (int c = nch; c >= 2; --c) {
      if (nch % c || c % 2) continue;
      const size_t slabs = 2 * (size_t)c * kPlane, blk = (size_t)c * cout * 16;
      if (slabs + 8 * blk > kConvSmemMax) continue;
      cc = c;
      ring = (int)std::min<size_t>(kMaxRing, (kConvSmemMax - slabs) / blk);
      break;
    }
  }
  if (!cc) return fail(VFLIP_ERR_ARG, "conv: no shared-memory split for %d -> %d", cin, cout);
  CUtensorMap amap;
  if (!make_map(&amap, in, X, Y, Z, kSX, kSY, 3)) return fail(VFLIP_ERR_CUDA, "conv: tensor map encode failed");
  ConvArgs a{};
  a.w = wpacked;
  a.bias = bias;
  a.mask = mask ? mask->p : nullptr;
  a.mstride = mask ? mask->ctot : 0;
  a.moff = mask ? mask->coff : 0;
  a.out = out ? out->p : nullptr;
  a.ostride = out ? out->ctot : 0;
  a.ooff = out ? out->coff : 0;
  a.outf = outf;
  a.ofstride = ofstride;
  a.ofvalid = ofvalid;
  a.X = X;
  a.Y = Y;
  a.Z = Z;
  a.cin = cin;
  a.cout = cout;
  a.cc = cc;
  a.ngroups = nch / cc;
  a.relu = relu;
  a.ntx = (X + kTX - 1) / kTX;
  a.nty = (Y + kTY - 1) / kTY;
  a.ntiles = a.ntx * a.nty * Z;
  a.ring = ring;
  a.lag = ring >= 27 * a.ngroups ? 0 : std::min(4, ring / 4);
  a.tmem_cols = pow2_cols(cout);
  a.error = d_error;
  const size_t smem = std::max(kConvSmemFloor, 2 * (size_t)cc * kPlane + (size_t)ring * cc * cout * 16);
  const int grid = std::min(a.ntiles, 2 * num_sms);
  conv3_tc_kernel<<<grid, kConvThreads, smem, stream>>>(amap, a);
  NET_LAUNCH();
  return VFLIP_OK;
}

int Net::wgrad(const View& x, const View& dy, int X, int Y, int Z, int cin, int cout, float* dw_master) {
  if (cin % 16 || cout % 16 || cout > 128) return fail(VFLIP_ERR_ARG, "wgrad: channels %d -> %d", cin, cout);
  if (!view_ok(x) || x.c != cin || !view_ok(dy) || dy.c != cout) return fail(VFLIP_ERR_ARG, "wgrad: bad views");
  const int nch = cin / 8;
  int cgn = 0;
  for (int c = std::min(nch, 8); c >= 2; --c)
    if (nch % c == 0 && c % 2 == 0 && 2 * ((size_t)16 * kDyPlane + (size_t)c * kPlane) <= kWgradSmemMax) {
      cgn = c;
      break;
    }
  if (!cgn) return fail(VFLIP_ERR_ARG, "wgrad: no shared-memory split");
  WgradArgs a{};
  a.X = X;
  a.Y = Y;
  a.Z = Z;
  a.cin = cin;
  a.cout = cout;
  a.ntx = (X + kTX - 1) / kTX;
  a.nty = (Y + kTY - 1) / kTY;
  a.ntiles = a.ntx * a.nty * Z;
  const int N = 8 * cgn;
  a.cgn = cgn;
  a.nng = nch / cgn;
  a.tpg = std::min(27, 512 / N);
  a.ntg = (27 + a.tpg - 1) / a.tpg;
  const int base = a.ntg * a.nng;
  int nsplit = std::max(1, std::min(a.ntiles, (num_sms + base - 1) / base));
  a.tiles_per_split = (a.ntiles + nsplit - 1) / nsplit;
  a.nsplit = (a.ntiles + a.tiles_per_split - 1) / a.tiles_per_split;
  a.tmem_cols = 512;
  a.error = d_error;
  const size_t n = (size_t)27 * cout * cin;
  a.partial = static_cast<float*>(scratch(sizeof(float) * n * a.nsplit, 0));
  if (!a.partial) return fail(VFLIP_ERR_NOMEM, "wgrad: workspace");
  CUtensorMap xmap, dymap;
  if (!make_map(&xmap, x, X, Y, Z, kSX, kSY, 3) || !make_map(&dymap, dy, X, Y, Z, kTX, kTY, 1))
    return fail(VFLIP_ERR_CUDA, "wgrad: tensor map encode failed");
  const size_t smem = std::max(kWgradSmemFloor, 2 * ((size_t)16 * kDyPlane + (size_t)cgn * kPlane));
  conv3_wgrad_tc_kernel<<<base * a.nsplit, kConvThreads, smem, stream>>>(xmap, dymap, a);
  NET_LAUNCH();
  wgrad_reduce_kernel<<<grid1(n, num_sms), 256, 0, stream>>>(a.partial, dw_master, a.nsplit, cin, cout);
  NET_LAUNCH();
  return VFLIP_OK;
}

int Net::channel_sum(const View& g, size_t nvox, float* out) {
  const size_t chunk = 2048;
  const int nb = (int)((nvox + chunk - 1) / chunk);
  float* part = static_cast<float*>(scratch(sizeof(float) * (size_t)nb * g.c, 1));
  if (!part) return fail(VFLIP_ERR_NOMEM, "channel sum workspace");
  channel_sum_partial_kernel<<<nb, 128, 0, stream>>>(g.p, g.ctot, g.coff, g.c, nvox, chunk, part);
  NET_LAUNCH();
  channel_sum_final_kernel<<<1, 256, 0, stream>>>(part, nb, g.c, out);
  NET_LAUNCH();
  return VFLIP_OK;
}

// ---------------------------------------------------------------- network
int Net::ensure_acts(int X, int Y, int Z) {
  if (X <= 0 || Y <= 0 || Z <= 0 || X % 8 || Y % 8 || Z % 8)
    return fail(VFLIP_ERR_ARG, "network grid %dx%dx%d: dimensions must be positive multiples of 8", X, Y, Z);
  if (acts && acts->X[0] == X && acts->Y[0] == Y && acts->Z[0] == Z) return VFLIP_OK;
  if (!acts) acts = new Acts();
  Acts& A = *acts;
  for (int l = 0; l < 4; ++l) {
    A.X[l] = X >> l;
    A.Y[l] = Y >> l;
    A.Z[l] = Z >> l;
    A.V[l] = (size_t)A.X[l] * A.Y[l] * A.Z[l];
  }
  struct Req {
    __nv_bfloat16** p;
    int level, c;
  };
  const Req reqs[] = {
      {&A.in0, 0, 16},    {&A.a_e0a, 0, 16},  {&A.cat0, 0, 48},   {&A.p1, 1, 16},     {&A.a_e1a, 1, 32},
      {&A.cat1, 1, 96},   {&A.p2, 2, 32},     {&A.a_e2a, 2, 64},  {&A.cat2, 2, 192},  {&A.p3, 3, 64},
      {&A.a_b1, 3, 128},  {&A.b3, 3, 128},    {&A.a_d2a, 2, 64},  {&A.d2, 2, 64},     {&A.a_d1a, 1, 32},
      {&A.d1, 1, 32},     {&A.a_d0a, 0, 16},  {&A.d0, 0, 16},     {&A.g_out, 0, 16},  {&A.g_d0, 0, 16},
      {&A.g_d0a, 0, 16},  {&A.g_cat0, 0, 48}, {&A.g_d1, 1, 32},   {&A.g_d1a, 1, 32},  {&A.g_cat1, 1, 96},
      {&A.g_d2, 2, 64},   {&A.g_d2a, 2, 64},  {&A.g_cat2, 2, 192}, {&A.g_b3, 3, 128}, {&A.g_b1, 3, 128},
      {&A.g_p3, 3, 64},   {&A.g_e2a, 2, 64},  {&A.g_p2, 2, 32},   {&A.g_e1a, 1, 32},  {&A.g_p1, 1, 16},
      {&A.g_e0a, 0, 16},
  };
  size_t bytes = 0;
  for (const Req& r : reqs) bytes += ((A.V[r.level] * r.c * 2 + 255) / 256) * 256;
  const size_t out_bytes = ((A.V[0] * 2 * sizeof(float) + 255) / 256) * 256;
  bytes += out_bytes;
  if (bytes > act_bytes) {
    cudaFree(act_mem);
    act_mem = nullptr;
    act_bytes = 0;
    if (cudaMalloc(&act_mem, bytes) != cudaSuccess) return fail(VFLIP_ERR_NOMEM, "network activations (%zu B)", bytes);
    act_bytes = bytes;
  }
  char* p = static_cast<char*>(act_mem);
  for (const Req& r : reqs) {
    *r.p = reinterpret_cast<__nv_bfloat16*>(p);
    p += ((A.V[r.level] * r.c * 2 + 255) / 256) * 256;
  }
  A.out2 = reinterpret_cast<float*>(p);
  // buffers read through halos or channel views before every channel is written start at zero
  NET_CUDA(cudaMemsetAsync(act_mem, 0, bytes, stream));
  A.have_forward = false;
  return VFLIP_OK;
}

namespace {
View V_(__nv_bfloat16* p, int ctot, int coff, int c) { return View{p, ctot, coff, c}; }
}  // namespace

int Net::forward(int X, int Y, int Z, const float* in2, float* out2) {
  NET_TRY(ensure_acts(X, Y, Z));
  NET_CUDA(cudaSetDevice(device));
  Acts& A = *acts;
  auto conv_l = [&](int l, int lev, const View& in, const View* out, float* of) {
    return conv(in, A.X[lev], A.Y[lev], A.Z[lev], wf[l], params + boff[l], kSpec[l].cin, kSpec[l].cout,
                kSpec[l].relu, nullptr, out, of, kOutValid, kOutValid);
  };
  pack_input_kernel<<<grid1(A.V[0], num_sms), 256, 0, stream>>>(in2, A.in0, A.V[0]);
  NET_LAUNCH();
  View v;
  NET_TRY(conv_l(E0A, 0, V_(A.in0, 16, 0, 16), &(v = V_(A.a_e0a, 16, 0, 16)), nullptr));
  NET_TRY(conv_l(E0B, 0, V_(A.a_e0a, 16, 0, 16), &(v = V_(A.cat0, 48, 32, 16)), nullptr));
  avgpool_kernel<<<grid1(A.V[1] * 2, num_sms), 256, 0, stream>>>(A.cat0, 48, 32, A.p1, 16, A.X[0], A.Y[0], A.Z[0]);
  NET_LAUNCH();
  NET_TRY(conv_l(E1A, 1, V_(A.p1, 16, 0, 16), &(v = V_(A.a_e1a, 32, 0, 32)), nullptr));
  NET_TRY(conv_l(E1B, 1, V_(A.a_e1a, 32, 0, 32), &(v = V_(A.cat1, 96, 64, 32)), nullptr));
  avgpool_kernel<<<grid1(A.V[2] * 4, num_sms), 256, 0, stream>>>(A.cat1, 96, 64, A.p2, 32, A.X[1], A.Y[1], A.Z[1]);
  NET_LAUNCH();
  NET_TRY(conv_l(E2A, 2, V_(A.p2, 32, 0, 32), &(v = V_(A.a_e2a, 64, 0, 64)), nullptr));
  NET_TRY(conv_l(E2B, 2, V_(A.a_e2a, 64, 0, 64), &(v = V_(A.cat2, 192, 128, 64)), nullptr));
  avgpool_kernel<<<grid1(A.V[3] * 8, num_sms), 256, 0, stream>>>(A.cat2, 192, 128, A.p3, 64, A.X[2], A.Y[2], A.Z[2]);
  NET_LAUNCH();
  NET_TRY(conv_l(B1, 3, V_(A.p3, 64, 0, 64), &(v = V_(A.a_b1, 128, 0, 128)), nullptr));
  NET_TRY(conv_l(B2, 3, V_(A.a_b1, 128, 0, 128), &(v = V_(A.b3, 128, 0, 128)), nullptr));
  upsample_kernel<<<grid1(A.V[2] * 16, num_sms), 256, 0, stream>>>(A.b3, A.cat2, 192, 128, A.X[2], A.Y[2], A.Z[2]);
  NET_LAUNCH();
  NET_TRY(conv_l(D2A, 2, V_(A.cat2, 192, 0, 192), &(v = V_(A.a_d2a, 64, 0, 64)), nullptr));
  NET_TRY(conv_l(D2B, 2, V_(A.a_d2a, 64, 0, 64), &(v = V_(A.d2, 64, 0, 64)), nullptr));
  upsample_kernel<<<grid1(A.V[1] * 8, num_sms), 256, 0, stream>>>(A.d2, A.cat1, 96, 64, A.X[1], A.Y[1], A.Z[1]);
  NET_LAUNCH();
  NET_TRY(conv_l(D1A, 1, V_(A.cat1, 96, 0, 96), &(v = V_(A.a_d1a, 32, 0, 32)), nullptr));
  NET_TRY(conv_l(D1B, 1, V_(A.a_d1a, 32, 0, 32), &(v = V_(A.d1, 32, 0, 32)), nullptr));
  upsample_kernel<<<grid1(A.V[0] * 4, num_sms), 256, 0, stream>>>(A.d1, A.cat0, 48, 32, A.X[0], A.Y[0], A.Z[0]);
  NET_LAUNCH();
  NET_TRY(conv_l(D0A, 0, V_(A.cat0, 48, 0, 48), &(v = V_(A.a_d0a, 16, 0, 16)), nullptr));
  NET_TRY(conv_l(D0B, 0, V_(A.a_d0a, 16, 0, 16), &(v = V_(A.d0, 16, 0, 16)), nullptr));
  NET_TRY(conv_l(OUT, 0, V_(A.d0, 16, 0, 16), nullptr, A.out2));
  if (out2 && out2 != A.out2) {
    NET_CUDA(cudaMemcpyAsync(out2, A.out2, A.V[0] * 2 * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  }
  A.have_forward = true;
  return VFLIP_OK;
}

int Net::forward_replay(int X, int Y, int Z, const float* in2, float* out2) {
  NET_TRY(ensure_acts(X, Y, Z));  // any allocation happens outside the capture
  NET_CUDA(cudaSetDevice(device));
  const std::vector<uintptr_t> key = {(uintptr_t)X, (uintptr_t)Y, (uintptr_t)Z, (uintptr_t)in2, (uintptr_t)out2,
                                      (uintptr_t)act_mem};
  if (!fwd_exec || key != fwd_key) {
    if (fwd_exec) cudaGraphExecDestroy(fwd_exec);
    if (fwd_graph) cudaGraphDestroy(fwd_graph);
    fwd_exec = nullptr;
    fwd_graph = nullptr;
    fwd_key.clear();
    if (!cap_stream) NET_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    NET_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
    const cudaStream_t saved = stream;
    const long long l0 = launches;
    stream = cap_stream;
    const int rc = forward(X, Y, Z, in2, out2);
    stream = saved;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cap_stream, &g);
    if (rc || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return rc ? rc : fail(VFLIP_ERR_CUDA, "network capture: %s", cudaGetErrorString(e));
    }
    fwd_graph = g;
    if (cudaGraphInstantiate(&fwd_exec, g, 0) != cudaSuccess) {
      fwd_exec = nullptr;
      return fail(VFLIP_ERR_CUDA, "network graph instantiate failed");
    }
    fwd_launches = launches - l0;
    launches = l0;  // captured launches count when the graph runs
    fwd_key = key;
  }
  NET_CUDA(cudaGraphLaunch(fwd_exec, stream));
  launches += fwd_launches;
  acts->have_forward = true;
  return VFLIP_OK;
}

int Net::backward(const float* target2, const float* weight, float cw0, float cw1, double* loss) {
  if (!acts || !acts->have_forward) return fail(VFLIP_ERR_ARG, "backward needs a forward pass first");
  Acts& A = *acts;
  NET_CUDA(cudaSetDevice(device));
  // loss and its gradient
  const int nb = std::min<int>(1024, grid1(A.V[0], num_sms));
  double* lp = static_cast<double*>(scratch(sizeof(double) * nb, 2));
  if (!lp) return fail(VFLIP_ERR_NOMEM, "loss workspace");
  const float inv_norm = 1.0f / (float)A.V[0];
  mse_loss_kernel<<<nb, 256, 0, stream>>>(A.out2, target2, weight, A.V[0], inv_norm, cw0, cw1, A.g_out, lp);
  NET_LAUNCH();
  NET_CUDA(cudaMemsetAsync(grads, 0, sizeof(float) * nparams, stream));

  // dz of layer l = `dz`; its input activation view `x`; dgrad into `dx` masked by `mask` (may be null)
  auto layer_bwd = [&](int l, int lev, const View& x, const View& dz, const View* dx, const View* mask) -> int {
    const int Xl = A.X[lev], Yl = A.Y[lev], Zl = A.Z[lev];
    NET_TRY(wgrad(x, dz, Xl, Yl, Zl, kSpec[l].cin, kSpec[l].cout, grads + woff[l]));
    NET_TRY(channel_sum(dz, A.V[lev], grads + boff[l]));
    if (dx) NET_TRY(conv(dz, Xl, Yl, Zl, wd[l], nullptr, kSpec[l].cout, kSpec[l].cin, 0, mask, dx, nullptr, 0, 0));
    return VFLIP_OK;
  };
  View dx, mk;
  NET_TRY(layer_bwd(OUT, 0, V_(A.d0, 16, 0, 16), V_(A.g_out, 16, 0, 16), &(dx = V_(A.g_d0, 16, 0, 16)),
                    &(mk = V_(A.d0, 16, 0, 16))));
  NET_TRY(layer_bwd(D0B, 0, V_(A.a_d0a, 16, 0, 16), V_(A.g_d0, 16, 0, 16), &(dx = V_(A.g_d0a, 16, 0, 16)),
                    &(mk = V_(A.a_d0a, 16, 0, 16))));
  NET_TRY(layer_bwd(D0A, 0, V_(A.cat0, 48, 0, 48), V_(A.g_d0a, 16, 0, 16), &(dx = V_(A.g_cat0, 48, 0, 48)),
                    &(mk = V_(A.cat0, 48, 0, 48))));
  upsample_bwd_kernel<<<grid1(A.V[1] * 4, num_sms), 256, 0, stream>>>(A.g_cat0, 48, A.g_d1, 32, A.X[0], A.Y[0],
                                                                        A.Z[0]);
  NET_LAUNCH();
  NET_TRY(layer_bwd(D1B, 1, V_(A.a_d1a, 32, 0, 32), V_(A.g_d1, 32, 0, 32), &(dx = V_(A.g_d1a, 32, 0, 32)),
                    &(mk = V_(A.a_d1a, 32, 0, 32))));
  NET_TRY(layer_bwd(D1A, 1, V_(A.cat1, 96, 0, 96), V_(A.g_d1a, 32, 0, 32), &(dx = V_(A.g_cat1, 96, 0, 96)),
                    &(mk = V_(A.cat1, 96, 0, 96))));
  upsample_bwd_kernel<<<grid1(A.V[2] * 8, num_sms), 256, 0, stream>>>(A.g_cat1, 96, A.g_d2, 64, A.X[1], A.Y[1],
                                                                        A.Z[1]);
  NET_LAUNCH();
  NET_TRY(layer_bwd(D2B, 2, V_(A.a_d2a, 64, 0, 64), V_(A.g_d2, 64, 0, 64), &(dx = V_(A.g_d2a, 64, 0, 64)),
                    &(mk = V_(A.a_d2a, 64, 0, 64))));
  NET_TRY(layer_bwd(D2A, 2, V_(A.cat2, 192, 0, 192), V_(A.g_d2a, 64, 0, 64), &(dx = V_(A.g_cat2, 192, 0, 192)),
                    &(mk = V_(A.cat2, 192, 0, 192))));
  upsample_bwd_kernel<<<grid1(A.V[3] * 16, num_sms), 256, 0, stream>>>(A.g_cat2, 192, A.g_b3, 128, A.X[2], A.Y[2],
                                                                         A.Z[2]);
  NET_LAUNCH();
  NET_TRY(layer_bwd(B2, 3, V_(A.a_b1, 128, 0, 128), V_(A.g_b3, 128, 0, 128), &(dx = V_(A.g_b1, 128, 0, 128)),
                    &(mk = V_(A.a_b1, 128, 0, 128))));
  NET_TRY(layer_bwd(B1, 3, V_(A.p3, 64, 0, 64), V_(A.g_b1, 128, 0, 128), &(dx = V_(A.g_p3, 64, 0, 64)), nullptr));
  avgpool_bwd_kernel<<<grid1(A.V[2] * 8, num_sms), 256, 0, stream>>>(A.g_p3, A.g_cat2, A.cat2, 192, 128, 64, A.X[2],
                                                                       A.Y[2], A.Z[2]);
  NET_LAUNCH();
  NET_TRY(layer_bwd(E2B, 2, V_(A.a_e2a, 64, 0, 64), V_(A.g_cat2, 192, 128, 64), &(dx = V_(A.g_e2a, 64, 0, 64)),
                    &(mk = V_(A.a_e2a, 64, 0, 64))));
  NET_TRY(layer_bwd(E2A, 2, V_(A.p2, 32, 0, 32), V_(A.g_e2a, 64, 0, 64), &(dx = V_(A.g_p2, 32, 0, 32)), nullptr));
  avgpool_bwd_kernel<<<grid1(A.V[1] * 4, num_sms), 256, 0, stream>>>(A.g_p2, A.g_cat1, A.cat1, 96, 64, 32, A.X[1],
                                                                       A.Y[1], A.Z[1]);
  NET_LAUNCH();
  NET_TRY(layer_bwd(E1B, 1, V_(A.a_e1a, 32, 0, 32), V_(A.g_cat1, 96, 64, 32), &(dx = V_(A.g_e1a, 32, 0, 32)),
                    &(mk = V_(A.a_e1a, 32, 0, 32))));
  NET_TRY(layer_bwd(E1A, 1, V_(A.p1, 16, 0, 16), V_(A.g_e1a, 32, 0, 32), &(dx = V_(A.g_p1, 16, 0, 16)), nullptr));
  avgpool_bwd_kernel<<<grid1(A.V[0] * 2, num_sms), 256, 0, stream>>>(A.g_p1, A.g_cat0, A.cat0, 48, 32, 16, A.X[0],
                                                                       A.Y[0], A.Z[0]);
  NET_LAUNCH();
  NET_TRY(layer_bwd(E0B, 0, V_(A.a_e0a, 16, 0, 16), V_(A.g_cat0, 48, 32, 16), &(dx = V_(A.g_e0a, 16, 0, 16)),
                    &(mk = V_(A.a_e0a, 16, 0, 16))));
  NET_TRY(layer_bwd(E0A, 0, V_(A.in0, 16, 0, 16), V_(A.g_e0a, 16, 0, 16), nullptr, nullptr));
  if (loss) {
    std::vector<double> h(nb);
    NET_CUDA(cudaMemcpyAsync(h.data(), lp, sizeof(double) * nb, cudaMemcpyDeviceToHost, stream));
    NET_CUDA(cudaStreamSynchronize(stream));
    double s = 0.0;
    for (double v : h) s += v;
    *loss = s;
  }
  return VFLIP_OK;
}

int Net::adam(float lr, float b1, float b2, float eps) {
  ++adam_t;
  const double c1 = 1.0 - std::pow((double)b1, adam_t), c2 = 1.0 - std::pow((double)b2, adam_t);
  const float lr_t = (float)(lr * std::sqrt(c2) / c1);
  adam_kernel<<<grid1((size_t)nparams, num_sms), 256, 0, stream>>>(params, grads, adam_m, adam_v, (size_t)nparams,
                                                                    lr_t, b1, b2, eps);
  NET_LAUNCH();
  return repack();
}

}  // namespace unet
}  // namespace vflip

// ---------------------------------------------------------------- C ABI
using vflip::unet::Net;
using vflip::unet::View;

extern "C" {

int vflip_unet_create(vflip_unet** out, int device, void* stream, unsigned long long seed) {
  if (!out) return VFLIP_ERR_ARG;
  *out = nullptr;
  vflip_unet* u = new vflip_unet{new Net(device, static_cast<cudaStream_t>(stream), seed)};
  *out = u;
  return u->net->init_status();
}

int vflip_unet_destroy(vflip_unet* u) {
  if (!u) return VFLIP_ERR_ARG;
  delete u->net;
  delete u;
  return VFLIP_OK;
}

const char* vflip_unet_last_error(const vflip_unet* u) { return u ? u->net->err.c_str() : "null network"; }

int vflip_unet_num_params(void) {
  size_t n = 0;
  for (int l = 0; l < vflip::unet::kNumLayers; ++l)
    n += (size_t)vflip::unet::kSpec[l].cout * (vflip::unet::kSpec[l].cin * 27 + 1);
  return (int)n;
}

int vflip_unet_get_params(vflip_unet* u, float* host) {
  if (!u || !host) return VFLIP_ERR_ARG;
  return u->net->get_params(host);
}

int vflip_unet_set_params(vflip_unet* u, const float* host) {
  if (!u || !host) return VFLIP_ERR_ARG;
  return u->net->set_params(host);
}

int vflip_unet_forward(vflip_unet* u, int X, int Y, int Z, const float* in2, float* out2) {
  if (!u || !in2) return VFLIP_ERR_ARG;
  int rc = u->net->forward_replay(X, Y, Z, in2, out2);
  if (rc) return rc;
  return u->net->sync_error();
}

int vflip_unet_gradients(vflip_unet* u, int X, int Y, int Z, const float* in2, const float* target2,
                         const float* weight, float cw0, float cw1, float* grad_out, double* loss) {
  if (!u || !in2 || !target2 || !weight) return VFLIP_ERR_ARG;
  Net& n = *u->net;
  int rc;
  if ((rc = n.forward(X, Y, Z, in2, nullptr))) return rc;
  if ((rc = n.backward(target2, weight, cw0, cw1, loss))) return rc;
  if (grad_out && (rc = n.copy_grads(grad_out))) return rc;
  return n.sync_error();
}

int vflip_unet_train_step(vflip_unet* u, int X, int Y, int Z, const float* in2, const float* target2,
                          const float* weight, float cw0, float cw1, float lr, double* loss) {
  if (!u || !in2 || !target2 || !weight || !(lr > 0.0f)) return VFLIP_ERR_ARG;
  Net& n = *u->net;
  int rc;
  if ((rc = n.forward(X, Y, Z, in2, nullptr))) return rc;
  if ((rc = n.backward(target2, weight, cw0, cw1, loss))) return rc;
  if ((rc = n.adam(lr))) return rc;
  return loss ? n.sync_error() : VFLIP_OK;
}

int vflip_unet_conv3(vflip_unet* u, int X, int Y, int Z, const void* in, int in_ctot, int in_coff, const float* w,
                     int layer_cin, int layer_cout, int backward_data, const float* bias, int relu, const void* mask,
                     int mask_ctot, int mask_coff, void* out, int out_ctot, int out_coff, float* outf, int outf_stride,
                     int outf_valid) {
  if (!u || !in || !w) return VFLIP_ERR_ARG;
  Net& n = *u->net;
  const int cin = backward_data ? layer_cout : layer_cin, cout = backward_data ? layer_cin : layer_cout;
  if (layer_cin <= 0 || layer_cout <= 0 || layer_cin % 16 || layer_cout % 16 || layer_cin > 256 || layer_cout > 256)
    return n.fail(VFLIP_ERR_ARG, "conv3: channels must be multiples of 16 in [16, 256]");
  __nv_bfloat16* wp = static_cast<__nv_bfloat16*>(n.scratch((size_t)27 * cin * cout * 2, 3));
  if (!wp) return n.fail(VFLIP_ERR_NOMEM, "conv3: packed weights");
  int rc;
  if ((rc = n.pack(w, wp, layer_cin, layer_cout, backward_data))) return rc;
  View vin{(__nv_bfloat16*)in, in_ctot, in_coff, cin};
  View vm{(__nv_bfloat16*)mask, mask_ctot, mask_coff, cout};
  View vo{(__nv_bfloat16*)out, out_ctot, out_coff, cout};
  if ((rc = n.conv(vin, X, Y, Z, wp, backward_data ? nullptr : bias, cin, cout, backward_data ? 0 : relu,
                   mask ? &vm : nullptr, out ? &vo : nullptr, outf, outf_stride, outf_valid)))
    return rc;
  return n.sync_error();
}

int vflip_unet_conv3_wgrad(vflip_unet* u, int X, int Y, int Z, const void* x, int x_ctot, int x_coff, int cin,
                           const void* dy, int dy_ctot, int dy_coff, int cout, float* dw) {
  if (!u || !x || !dy || !dw) return VFLIP_ERR_ARG;
  Net& n = *u->net;
  View vx{(__nv_bfloat16*)x, x_ctot, x_coff, cin};
  View vd{(__nv_bfloat16*)dy, dy_ctot, dy_coff, cout};
  int rc;
  if ((rc = n.wgrad(vx, vd, X, Y, Z, cin, cout, dw))) return rc;
  return n.sync_error();
}

long long vflip_unet_launch_count(const vflip_unet* u) { return u ? u->net->launches : 0; }

int vflip_unet_set_output_scale(vflip_unet* u, float s0, float s1) {
  if (!u || !(s0 > 0.0f) || !(s1 > 0.0f)) return VFLIP_ERR_ARG;
  u->net->out_scale[0] = s0;
  u->net->out_scale[1] = s1;
  return VFLIP_OK;
}

}  // extern "C"
