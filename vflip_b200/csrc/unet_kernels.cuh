// 3x3x3 convolutions of the learned preconditioner on the 5th-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulation in TMEM), plus the
// small elementwise kernels of the network (pooling, upsampling, packing,
// loss, Adam).
//
// Activations are channels-last BF16, [z][y][x][C], C a multiple of 8; a
// "view" is a channel range [coff, coff+cin) of a tensor with Ctot channels
// (the skip connections write straight into the decoder's concatenation
// buffers).
//
// Forward / backward-data convolution = implicit GEMM
//     D[m = voxel][n = c_out] = sum_{tap, c_in} A[voxel + tap][c_in] * W[tap][c_out][c_in]
// One CTA (128 threads) computes persistent output tiles of 8 (x) x 16 (y)
// voxels of one z plane (M = 128).  The 10 x 18 x 3 input slab around a tile
// is brought into shared memory by TMA, one 8-channel plane per tensor load,
// as [chunk][z][y][x][8 channels]: in the no-swizzle K-major canonical layout
// a row (voxel) is 16 bytes, rows 8 apart in x are one core matrix and the
// y rows are 160 bytes apart, so the A operand of every tap is the same slab
// with a shifted start address - the 27 taps reuse one copy of the input.
// Weights stay resident in shared memory when all 27 taps fit; otherwise
// they stream per tap through a ring of bulk copies.  One thread
// issues all copies and MMAs; the four warps then read the 128 x c_out
// accumulator from TMEM (warp w owns TMEM lanes 32w..32w+31) and apply the
// fused epilogue (bias, ReLU, or the ReLU-derivative mask of the backward
// pass) before storing BF16 and/or FP32.
//
// Backward-weight convolution
//     dW[tap][c_out][c_in] = sum_voxel dY[voxel][c_out] * X[voxel + tap][c_in]
// reduces over voxels, so voxels are the K dimension: both operands are
// MN-major (channels contiguous), A = dY tile (M = c_out padded to 128 with
// zero planes), B = the same shifted input slab, one TMEM accumulator of c_in
// columns per tap.  CTAs own (tap group, c_in group, voxel range) and write
// FP32 partial sums that a second kernel adds in a fixed order.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"
#include "sm100.cuh"

namespace vflip {
namespace unet {

constexpr int kTX = 8, kTY = 16;                  // output tile: 8 x 16 voxels of one z plane
constexpr int kSX = kTX + 2, kSY = kTY + 2;       // slab incl. 1-voxel halo (z: 3 planes)
constexpr uint32_t kSlabBox = (uint32_t)kSX * kSY * 3 * 16;  // bytes one slab-plane tensor load delivers
constexpr uint32_t kPlane = 8704;                 // slab plane stride in shared memory: 8640 B padded to 128 B
constexpr uint32_t kRowY = kSX * 16;              // bytes between slab rows in y
constexpr uint32_t kDyPlane = 128 * 16;           // one 8-channel plane of a dY tile
constexpr int kConvThreads = 128;
constexpr int kMaxRing = 32;                      // weight ring slots (runtime depth <= this)

__host__ __device__ constexpr uint32_t tap_shift(int tap) {
  return (uint32_t)((((tap / 9) * kSY + (tap / 3) % 3) * kSX + tap % 3) * 16);
}

struct ConvArgs {
  const __nv_bfloat16* w;  // packed weights [27][cin/8][cout][8]
  const float* bias;       // [cout] or null
  const __nv_bfloat16* mask;  // keep where mask > 0 (ReLU derivative) or null
  int mstride, moff;
  __nv_bfloat16* out;  // BF16 output view or null
  int ostride, ooff;
  float* outf;  // FP32 output (first ofvalid channels) or null
  int ofstride, ofvalid;
  int X, Y, Z, cin, cout, cc, ngroups, relu;
  int ntx, nty, ntiles;
  int ring, lag;  // weight slots and MMA steps kept queued; ring == 27 * ngroups: resident
  uint32_t tmem_cols;
  int* error;
};

__device__ __forceinline__ void store_bf16x16(__nv_bfloat16* dst, const float (&v)[16]) {
  uint32_t p[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    p[q] = *reinterpret_cast<uint32_t*>(&h);
  }
  uint4* d = reinterpret_cast<uint4*>(dst);
  d[0] = make_uint4(p[0], p[1], p[2], p[3]);
  d[1] = make_uint4(p[4], p[5], p[6], p[7]);
}

__device__ __forceinline__ void load_bf16x16(const __nv_bfloat16* src, float (&v)[16]) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4 u[2] = {s[0], s[1]};
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(u);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    float2 f = __bfloat1622float2(h[q]);
    v[2 * q] = f.x;
    v[2 * q + 1] = f.y;
  }
}

__global__ void __launch_bounds__(kConvThreads, 1) conv3_tc_kernel(const __grid_constant__ CUtensorMap amap,
                                                                     const ConvArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[6 + 2 * kMaxRing];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cc = a.cc, cout = a.cout, G = a.ngroups, R = a.ring, L = a.lag;
  const int steps_tile = G * 27;
  const bool resident = R >= steps_tile;
  const uint32_t sb = smem_u32(smem);
  const uint32_t slab_bytes = (uint32_t)cc * kPlane;
  const uint32_t bblk = (uint32_t)cc * cout * 16;
  const uint32_t ring0 = sb + 2 * slab_bytes;
  const uint32_t bar0 = smem_u32(bars);
  // barriers: 0-1 slab full, 2-3 slab free, accumulator full, drain, then R weight-full, R weight-free
  const uint32_t ACC_FULL = bar0 + 32u, DRAIN = bar0 + 40u;
  auto slab_full = [&](int b) { return bar0 + 8u * b; };
  auto slab_free = [&](int b) { return bar0 + 8u * (2 + b); };
  auto b_full = [&](int r) { return bar0 + 8u * (6 + r); };
  auto b_free = [&](int r) { return bar0 + 8u * (6 + R + r); };

  if (tid == 0) {
    for (int q = 0; q < 6 + 2 * R; ++q) mbar_init(bar0 + 8u * q, 1);
    mbar_init_fence();
    abort_sh = 0;
  }
  if (warp == 0) tmem_alloc(smem_u32(&tmem_sh), a.tmem_cols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  const int ntiles_me = (int)blockIdx.x < a.ntiles ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const long total_steps = (long)ntiles_me * steps_tile;
  const int total_slabs = ntiles_me * G;
  const int nch = a.cin >> 3;
  const uint32_t idesc = umma_idesc_bf16(128, cout, 0, 0);

  auto tile_of = [&](int it, int& tx, int& ty, int& tz) {
    const int t = (int)blockIdx.x + it * (int)gridDim.x;
    tx = t % a.ntx;
    const int r = t / a.ntx;
    ty = r % a.nty;
    tz = r / a.nty;
  };
  // producer state (thread 0)
  long b_issued = 0, b_done = 0;
  int s_issued = 0, s_done = 0;
  auto issue_slab = [&](int q) {
    int tx, ty, tz;
    tile_of(q / G, tx, ty, tz);
    const int g = q % G, buf = q & 1;
    mbar_expect_tx(slab_full(buf), (uint32_t)cc * kSlabBox);
    for (int k = 0; k < cc; ++k)
      tma_tile_4d(sb + buf * slab_bytes + k * kPlane, &amap, 8 * (g * cc + k), tx * kTX - 1, ty * kTY - 1, tz - 1,
                  slab_full(buf));
    s_issued = q + 1;
  };
  auto issue_w = [&](long s) {
    const int r = (int)(s % R);
    const int blk = (int)(s % steps_tile);  // g * 27 + tap
    const int g = blk / 27, tap = blk % 27;
    mbar_expect_tx(b_full(r), bblk);
    tma_bulk_g2s(ring0 + r * bblk, a.w + ((size_t)tap * nch + (size_t)g * cc) * cout * 8, bblk, b_full(r));
    b_issued = s + 1;
  };

  bool ok = true;
  if (tid == 0 && total_steps > 0) {
    issue_slab(0);
    const long pre = resident ? steps_tile : R - L;
    for (long p = 0; p < pre && p < total_steps; ++p) issue_w(p);
  }
  long s = 0;
  int q = 0;
  for (int it = 0; it < ntiles_me; ++it) {
    if (tid == 0) {
      for (int g = 0; g < G && ok; ++g, ++q) {
        const int buf = q & 1;
        ok = mbar_wait_bounded(slab_full(buf), (uint32_t)((q >> 1) & 1));
        if (!ok) break;
        s_done = q + 1;
        tc_fence_after();
        const uint32_t slab = sb + buf * slab_bytes;
        for (int tap = 0; tap < 27; ++tap, ++s) {
          const int r = (int)(s % R);
          if (!resident || s < R) {
            ok = mbar_wait_bounded(b_full(r), (uint32_t)((s / R) & 1));
            if (!ok) break;
            b_done = s + 1;
          }
          const uint32_t a0 = slab + tap_shift(tap), b0 = ring0 + r * bblk;
          for (int j = 0; j < (cc >> 1); ++j) {
            const uint64_t ad = umma_sdesc(a0 + 2u * j * kPlane, kPlane, kRowY);
            const uint64_t bd = umma_sdesc(b0 + 2u * j * cout * 16, cout * 16, 128);
            umma_bf16(tmem, ad, bd, idesc, (g | tap | j) != 0);
          }
          if (!resident) {
            umma_commit(b_free(r));
            const long nxt = s + (R - L);
            if (nxt < total_steps) {
              if (s >= L) {
                ok = mbar_wait_bounded(b_free((int)((s - L) % R)), (uint32_t)(((s - L) / R) & 1));
                if (!ok) break;
              }
              issue_w(nxt);
            }
          }
        }
        if (!ok) break;
        umma_commit(slab_free(buf));
        if (q + 1 < total_slabs) {
          if (q >= 1) {
            ok = mbar_wait_bounded(slab_free(buf ^ 1), (uint32_t)(((q - 1) >> 1) & 1));
            if (!ok) break;
          }
          issue_slab(q + 1);
        }
      }
      if (ok) {
        umma_commit(ACC_FULL);
      } else {
        abort_sh = 1;
        mbar_arrive(ACC_FULL);
      }
    }
    // the producer's own warp parks here instead of spinning beside it
    __syncwarp();
    const bool got = mbar_wait_bounded(ACC_FULL, (uint32_t)(it & 1));
    if (__syncthreads_or(!got || abort_sh)) {
      if (tid == 0) atomicExch(a.error, 1);
      break;
    }
    tc_fence_after();
    int tx, ty, tz;
    tile_of(it, tx, ty, tz);
    const int m = warp * 32 + lane;
    const int x = tx * kTX + (m & 7), y = ty * kTY + (m >> 3);
    const bool valid = x < a.X && y < a.Y;
    const size_t vox = ((size_t)tz * a.Y + (valid ? y : 0)) * a.X + (valid ? x : 0);
    for (int c0 = 0; c0 < cout; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (valid) {
        if (a.bias) {
#pragma unroll
          for (int k = 0; k < 16; ++k) v[k] += a.bias[c0 + k];
        }
        if (a.relu) {
#pragma unroll
          for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k], 0.0f);
        }
        if (a.mask) {
          float mk[16];
          load_bf16x16(a.mask + vox * a.mstride + a.moff + c0, mk);
#pragma unroll
          for (int k = 0; k < 16; ++k) v[k] = mk[k] > 0.0f ? v[k] : 0.0f;
        }
        if (a.out) store_bf16x16(a.out + vox * a.ostride + a.ooff + c0, v);
        if (a.outf) {
#pragma unroll
          for (int k = 0; k < 16; ++k)
            if (c0 + k < a.ofvalid) a.outf[vox * a.ofstride + c0 + k] = v[k];
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  // on an abort, or when copies are still in flight, wait (bounded) for
  // every copy and MMA before the shared memory goes away
  if (tid == 0 && (abort_sh || b_done < b_issued || s_done < s_issued)) {
    umma_commit(DRAIN);
    mbar_wait_bounded(DRAIN, 0);
    for (long p = b_done; p < b_issued; ++p) mbar_wait_bounded(b_full((int)(p % R)), (uint32_t)((p / R) & 1));
    for (int p = s_done; p < s_issued; ++p) mbar_wait_bounded(slab_full(p & 1), (uint32_t)((p >> 1) & 1));
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, a.tmem_cols);
}

// ---------------------------------------------------------------------------
// backward-weight convolution

struct WgradArgs {
  float* partial;  // [nsplit][27][cout][cin]
  int X, Y, Z, cin, cout;
  int ntx, nty, ntiles;
  int tpg, ntg;    // taps per tap group, number of tap groups
  int cgn, nng;    // 8-channel c_in planes per N group, number of N groups
  int nsplit, tiles_per_split;
  uint32_t tmem_cols;
  int* error;
};

__global__ void __launch_bounds__(kConvThreads, 1) conv3_wgrad_tc_kernel(const __grid_constant__ CUtensorMap xmap,
                                                                           const __grid_constant__ CUtensorMap dymap,
                                                                           const WgradArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[6];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int item = blockIdx.x;
  const int tg = item % a.ntg;
  item /= a.ntg;
  const int ng = item % a.nng;
  const int sp = item / a.nng;
  const int tap0 = tg * a.tpg, ntap = min(a.tpg, 27 - tap0);
  const int N = a.cgn * 8;
  const int t_begin = sp * a.tiles_per_split, t_end = min(a.ntiles, t_begin + a.tiles_per_split);
  const int nt = max(0, t_end - t_begin);
  const int dy_planes = a.cout >> 3;
  const uint32_t sb = smem_u32(smem);
  // per buffer: 16 dY planes (M = 128 rows of c_out, zero beyond cout) then cgn slab planes
  const uint32_t dy_bytes = 16u * kDyPlane, slab_bytes = (uint32_t)a.cgn * kPlane;
  const uint32_t buf_bytes = dy_bytes + slab_bytes;
  const uint32_t load_bytes = (uint32_t)dy_planes * kDyPlane + (uint32_t)a.cgn * kSlabBox;
  const uint32_t bar0 = smem_u32(bars);
  auto full = [&](int b) { return bar0 + 8u * b; };
  auto freeb = [&](int b) { return bar0 + 8u * (2 + b); };
  const uint32_t ACC_FULL = bar0 + 32u, DRAIN = bar0 + 40u;

  // zero the padding planes of both dY buffers (rows c_out..127 of A)
  for (int b = 0; b < 2; ++b) {
    uint4* z = reinterpret_cast<uint4*>(smem + b * buf_bytes + dy_planes * kDyPlane);
    const int n16 = (16 - dy_planes) * (int)(kDyPlane / 16);
    for (int e = tid; e < n16; e += blockDim.x) z[e] = make_uint4(0, 0, 0, 0);
  }
  fence_proxy_async();
  if (tid == 0) {
    for (int q = 0; q < 6; ++q) mbar_init(bar0 + 8u * q, 1);
    mbar_init_fence();
    abort_sh = 0;
  }
  if (warp == 0) tmem_alloc(smem_u32(&tmem_sh), a.tmem_cols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;
  const uint32_t idesc = umma_idesc_bf16(128, N, 1, 1);

  int issued = 0, done = 0;
  auto issue = [&](int i) {
    const int t = t_begin + i, b = i & 1;
    const int tx = t % a.ntx, r = t / a.ntx, ty = r % a.nty, tz = r / a.nty;
    const uint32_t base = sb + b * buf_bytes;
    mbar_expect_tx(full(b), load_bytes);
    for (int k = 0; k < dy_planes; ++k) tma_tile_4d(base + k * kDyPlane, &dymap, 8 * k, tx * kTX, ty * kTY, tz, full(b));
    for (int k = 0; k < a.cgn; ++k)
      tma_tile_4d(base + dy_bytes + k * kPlane, &xmap, 8 * (ng * a.cgn + k), tx * kTX - 1, ty * kTY - 1, tz - 1,
                  full(b));
    issued = i + 1;
  };
  bool ok = true;
  if (tid == 0) {
    if (nt > 0) issue(0);
    for (int i = 0; i < nt && ok; ++i) {
      const int b = i & 1;
      ok = mbar_wait_bounded(full(b), (uint32_t)((i >> 1) & 1));
      if (!ok) break;
      done = i + 1;
      tc_fence_after();
      const uint32_t abase = sb + b * buf_bytes, xbase = abase + dy_bytes;
      for (int tl = 0; tl < ntap; ++tl) {
        const uint32_t xs = xbase + tap_shift(tap0 + tl);
        for (int kk = 0; kk < 8; ++kk) {  // 16 voxels (two y rows of the tile) per MMA
          const uint64_t ad = umma_sdesc(abase + kk * 256u, 128u, kDyPlane);
          const uint64_t bd = umma_sdesc(xs + kk * 2u * kRowY, kRowY, kPlane);
          umma_bf16(tmem + (uint32_t)(tl * N), ad, bd, idesc, (i | kk) != 0);
        }
      }
      umma_commit(freeb(b));
      if (i + 1 < nt) {
        if (i >= 1) {
          ok = mbar_wait_bounded(freeb(b ^ 1), (uint32_t)(((i - 1) >> 1) & 1));
          if (!ok) break;
        }
        issue(i + 1);
      }
    }
    if (ok) {
      umma_commit(ACC_FULL);
    } else {
      abort_sh = 1;
      mbar_arrive(ACC_FULL);
    }
  }
  __syncwarp();
  const bool got = mbar_wait_bounded(ACC_FULL, 0);
  if (__syncthreads_or(!got || abort_sh)) {
    if (tid == 0) {
      atomicExch(a.error, 1);
      umma_commit(DRAIN);
      mbar_wait_bounded(DRAIN, 0);
      for (int p = done; p < issued; ++p) mbar_wait_bounded(full(p & 1), (uint32_t)((p >> 1) & 1));
    }
  } else {
    tc_fence_after();
    const int co = warp * 32 + lane;  // TMEM lane = row of D = c_out
    for (int tl = 0; tl < ntap; ++tl) {
      for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(tl * N + c0), v);
        if (co < a.cout) {
          float* dst = a.partial + (((size_t)sp * 27 + tap0 + tl) * a.cout + co) * a.cin + ng * N + c0;
#pragma unroll
          for (int k = 0; k < 16; k += 4) *reinterpret_cast<float4*>(dst + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, a.tmem_cols);
}

// dW in the master layout [co][ci][tap] = sum over the splits' partials
// [split][tap][co][ci], splits in ascending order (deterministic)
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, float* __restrict__ dw, int nsplit, int cin,
                                    int cout) {
  const size_t n = (size_t)27 * cin * cout;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int tap = (int)(e % 27);
    const size_t r = e / 27;
    const int ci = (int)(r % cin), co = (int)(r / cin);
    const size_t src = ((size_t)tap * cout + co) * cin + ci;
    float s = 0.0f;
    for (int p = 0; p < nsplit; ++p) s += partial[(size_t)p * n + src];
    dw[e] = s;
  }
}

}  // namespace unet
}  // namespace vflip

namespace vflip {
namespace unet {

// ---------------------------------------------------------------------------
// elementwise kernels (grid-stride; channels-last BF16 views)

// master FP32 weights [cout][cin][27] -> packed BF16 [27][cin/8][cout][8]
// (flip = 0), or the backward-data weights of the same layer, a convolution
// from cout to cin channels with the taps mirrored (flip = 1):
// [27][cout/8][cin][8], element (t', co, ci) = W[co][ci][26 - t'].
__global__ void pack_weights_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ out, int cin, int cout,
                                    int flip) {
  const size_t n = (size_t)27 * cin * cout;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    // e enumerates the packed output
    const int lo = (int)(e % 8);
    size_t r = e / 8;
    if (!flip) {
      const int co = (int)(r % cout);
      r /= cout;
      const int chunk = (int)(r % (cin / 8));
      const int tap = (int)(r / (cin / 8));
      const int ci = chunk * 8 + lo;
      out[e] = __float2bfloat16_rn(w[((size_t)co * cin + ci) * 27 + tap]);
    } else {
      const int ci = (int)(r % cin);
      r /= cin;
      const int chunk = (int)(r % (cout / 8));
      const int tap = (int)(r / (cout / 8));
      const int co = chunk * 8 + lo;
      out[e] = __float2bfloat16_rn(w[((size_t)co * cin + ci) * 27 + (26 - tap)]);
    }
  }
}

// network input: channel 0 = scale * rhs, channel 1 = fluid mask, 2..15 = 0
__global__ void pack_input_kernel(const float* __restrict__ in2, __nv_bfloat16* __restrict__ out, size_t nvox) {
  for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (size_t)gridDim.x * blockDim.x) {
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = 0.0f;
    f[0] = in2[2 * v];
    f[1] = in2[2 * v + 1];
    store_bf16x16(out + v * 16, f);
  }
}

// 2x2x2 average pooling of a view (C channels at offset ioff of istride)
// into a dense [.][C] tensor; one thread per (coarse voxel, 8 channels)
__global__ void avgpool_kernel(const __nv_bfloat16* __restrict__ in, int istride, int ioff,
                               __nv_bfloat16* __restrict__ out, int C, int X, int Y, int Z) {
  const int cx = X / 2, cy = Y / 2, cz = Z / 2, c8 = C / 8;
  const size_t n = (size_t)cx * cy * cz * c8;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c8) * 8;
    size_t r = e / c8;
    const int i = (int)(r % cx), j = (int)((r / cx) % cy), k = (int)(r / ((size_t)cx * cy));
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int d = 0; d < 8; ++d) {
      const size_t v = ((size_t)(2 * k + (d >> 2)) * Y + 2 * j + ((d >> 1) & 1)) * X + 2 * i + (d & 1);
      const uint4 u = *reinterpret_cast<const uint4*>(in + v * istride + ioff + ch);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float2 f = __bfloat1622float2(h[q]);
        s[2 * q] += f.x;
        s[2 * q + 1] += f.y;
      }
    }
    uint32_t p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      __nv_bfloat162 h = __floats2bfloat162_rn(0.125f * s[2 * q], 0.125f * s[2 * q + 1]);
      p[q] = *reinterpret_cast<uint32_t*>(&h);
    }
    *reinterpret_cast<uint4*>(out + r * C + ch) = make_uint4(p[0], p[1], p[2], p[3]);
  }
}

// backward of avgpool, accumulated into the gradient view of its input and
// masked by the ReLU derivative of that input: g[child] += (a[child] > 0) dp/8
__global__ void avgpool_bwd_kernel(const __nv_bfloat16* __restrict__ dp, __nv_bfloat16* __restrict__ g,
                                   const __nv_bfloat16* __restrict__ act, int stride, int off, int C, int X, int Y,
                                   int Z) {
  const int c8 = C / 8;
  const size_t n = (size_t)X * Y * Z * c8;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c8) * 8;
    const size_t v = e / c8;
    const int i = (int)(v % X), j = (int)((v / X) % Y), k = (int)(v / ((size_t)X * Y));
    const size_t pv = ((size_t)(k / 2) * (Y / 2) + j / 2) * (X / 2) + i / 2;
    const uint4 ud = *reinterpret_cast<const uint4*>(dp + pv * C + ch);
    const uint4 ua = *reinterpret_cast<const uint4*>(act + v * stride + off + ch);
    uint4* gp = reinterpret_cast<uint4*>(g + v * stride + off + ch);
    uint4 ug = *gp;
    const __nv_bfloat162* hd = reinterpret_cast<const __nv_bfloat162*>(&ud);
    const __nv_bfloat162* ha = reinterpret_cast<const __nv_bfloat162*>(&ua);
    __nv_bfloat162* hg = reinterpret_cast<__nv_bfloat162*>(&ug);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float2 d = __bfloat1622float2(hd[q]), a = __bfloat1622float2(ha[q]), o = __bfloat1622float2(hg[q]);
      hg[q] = __floats2bfloat162_rn(o.x + (a.x > 0.0f ? 0.125f * d.x : 0.0f), o.y + (a.y > 0.0f ? 0.125f * d.y : 0.0f));
    }
    *gp = ug;
  }
}

// nearest 2x upsampling of a dense [.][C] tensor into channels [0, C) of a
// view with stride ostride (the decoder's concatenation buffer)
__global__ void upsample_kernel(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, int ostride,
                                int C, int X, int Y, int Z) {
  const int c8 = C / 8;
  const size_t n = (size_t)X * Y * Z * c8;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c8) * 8;
    const size_t v = e / c8;
    const int i = (int)(v % X), j = (int)((v / X) % Y), k = (int)(v / ((size_t)X * Y));
    const size_t pv = ((size_t)(k / 2) * (Y / 2) + j / 2) * (X / 2) + i / 2;
    *reinterpret_cast<uint4*>(out + v * ostride + ch) = *reinterpret_cast<const uint4*>(in + pv * C + ch);
  }
}

// backward of upsample: the gradient of a coarse voxel is the sum over its 8
// children (already masked by the ReLU derivative in the producing epilogue)
__global__ void upsample_bwd_kernel(const __nv_bfloat16* __restrict__ g, int gstride,
                                    __nv_bfloat16* __restrict__ out, int C, int X, int Y, int Z) {
  const int cx = X / 2, cy = Y / 2, cz = Z / 2, c8 = C / 8;
  const size_t n = (size_t)cx * cy * cz * c8;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c8) * 8;
    size_t r = e / c8;
    const int i = (int)(r % cx), j = (int)((r / cx) % cy), k = (int)(r / ((size_t)cx * cy));
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int d = 0; d < 8; ++d) {
      const size_t v = ((size_t)(2 * k + (d >> 2)) * Y + 2 * j + ((d >> 1) & 1)) * X + 2 * i + (d & 1);
      const uint4 u = *reinterpret_cast<const uint4*>(g + v * gstride + ch);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float2 f = __bfloat1622float2(h[q]);
        s[2 * q] += f.x;
        s[2 * q + 1] += f.y;
      }
    }
    uint32_t p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      __nv_bfloat162 h = __floats2bfloat162_rn(s[2 * q], s[2 * q + 1]);
      p[q] = *reinterpret_cast<uint32_t*>(&h);
    }
    *reinterpret_cast<uint4*>(out + r * C + ch) = make_uint4(p[0], p[1], p[2], p[3]);
  }
}

// weighted MSE over the two output channels: per-block partial losses and
// the output gradient 2 w (o - t) / norm in channels 0-1 of a 16-channel
// BF16 tensor (channels 2-15 zero)
__global__ void mse_loss_kernel(const float* __restrict__ out2, const float* __restrict__ t2,
                                const float* __restrict__ w, size_t nvox, float inv_norm, float cw0, float cw1,
                                __nv_bfloat16* __restrict__ grad, double* __restrict__ partial) {
  __shared__ double red[32];
  double acc = 0.0;
  for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (size_t)gridDim.x * blockDim.x) {
    const float wv = w[v];
    const float d0 = out2[2 * v] - t2[2 * v], d1 = out2[2 * v + 1] - t2[2 * v + 1];
    acc += (double)(wv * (cw0 * d0 * d0 + cw1 * d1 * d1));
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = 0.0f;
    f[0] = 2.0f * wv * cw0 * d0 * inv_norm;
    f[1] = 2.0f * wv * cw1 * d1 * inv_norm;
    store_bf16x16(grad + v * 16, f);
  }
  acc = block_sum<256>(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc * (double)inv_norm;
}

// per-channel sums of a view over all voxels: block b sums voxels
// [b*chunk, (b+1)*chunk) into partial[b][C]; ascending order, deterministic
__global__ void channel_sum_partial_kernel(const __nv_bfloat16* __restrict__ g, int stride, int off, int C,
                                           size_t nvox, size_t chunk, float* __restrict__ partial) {
  const size_t v0 = blockIdx.x * chunk, v1 = min(nvox, v0 + chunk);
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    float s = 0.0f;
    for (size_t v = v0; v < v1; ++v) s += __bfloat162float(g[v * stride + off + c]);
    partial[(size_t)blockIdx.x * C + c] = s;
  }
}
__global__ void channel_sum_final_kernel(const float* __restrict__ partial, int nb, int C, float* __restrict__ out) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int b = 0; b < nb; ++b) s += partial[(size_t)b * C + c];
    out[c] = s;
  }
}

// Adam on the FP32 master parameters (bias-corrected step sizes on the host)
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr_t, float b1, float b2, float eps) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.0f - b1) * gi;
    const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    p[e] -= lr_t * mi / (sqrtf(vi) + eps);
  }
}

}  // namespace unet
}  // namespace vflip
