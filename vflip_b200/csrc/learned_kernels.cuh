// Kernels of the learned-preconditioned solve: the network's features on a
// coarse grid (block averages of the rhs and of the fluid indicator, scaled
// by 1/|rhs_c|_inf), the trilinear prolongation of its two outputs back to
// the fine grid, the Ritz step over the initial subspace, and the flexible
// (Polak-Ribiere) PCG update.  No reference counterpart.
#pragma once
#include "common.cuh"
#include "pcg_kernels.cuh"

namespace vflip {

// Network grid of a fine grid at multigrid level L: ceil(n / 2^L) rounded up
// to a multiple of 8 (the network pools three times).
inline void learned_grid_dims(int ni, int nj, int nk, int L, int& X, int& Y, int& Z) {
  auto f = [L](int n) {
    const int c = (n + (1 << L) - 1) >> L;
    return (c + 7) / 8 * 8;
  };
  X = f(ni);
  Y = f(nj);
  Z = f(nk);
}

// out[v] (network grid X x Y x Z) = (1/8^L) * sum over the fine cells of the
// 2^L block of f(a, b); blocks beyond the fine grid are 0.  This is R^L of
// the multigrid restriction (out-of-range children add nothing).
//   kind 0: a;  kind 1: (a > 0) (fluid indicator of the diagonal);  kind 2: a - b
template <typename TA, typename TB>
__global__ void block_average_kernel(const TA* __restrict__ a, const TB* __restrict__ b, int kind, int ni, int nj,
                                     int nk, int L, float* __restrict__ out, int X, int Y, int Z) {
  const size_t nv = (size_t)X * Y * Z;
  const int B = 1 << L;
  const double inv = 1.0 / (double)((size_t)B * B * B);
  for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
    const int I = (int)(v % X), J = (int)((v / X) % Y), K = (int)(v / ((size_t)X * Y));
    double s = 0.0;
    for (int k = K * B; k < min(nk, (K + 1) * B); ++k)
      for (int j = J * B; j < min(nj, (J + 1) * B); ++j)
        for (int i = I * B; i < min(ni, (I + 1) * B); ++i) {
          const size_t e = lin3(i, j, k, ni, nj);
          const double va = (double)a[e];
          s += kind == 0 ? va : kind == 1 ? (va > 0.0 ? 1.0 : 0.0) : va - (double)b[e];
        }
    out[v] = (float)(s * inv);
  }
}

// partial max |f| per block, folded by the last block into *scale = 1/max (0 if max == 0)
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) inv_absmax_kernel(const float* __restrict__ f, size_t n, double* partials,
                                                           unsigned int* counter, double* scale) {
  __shared__ double sm[BLOCK / 32];
  __shared__ bool last;
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK)
    m = fmax(m, fabs((double)f[i]));
  m = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = m;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += BLOCK) v = fmax(v, ((volatile double*)partials)[q]);
  v = block_absmax<BLOCK>(v, sm);
  if (threadIdx.x == 0) {
    *scale = v > 0.0 ? 1.0 / v : 0.0;
    *counter = 0;
  }
}

// out2[v] = (scale * c0[v], c1 ? scale1 * c1[v] : w[v]) packs two channels
__global__ void pack2_kernel(const float* __restrict__ c0, const float* __restrict__ c1, const double* __restrict__ scale,
                             int scale_c1, float* __restrict__ out2, size_t n) {
  const float s = (float)*scale;
  for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x) {
    out2[2 * v] = s * c0[v];
    out2[2 * v + 1] = scale_c1 ? s * c1[v] : c1[v];
  }
}

// w[fine] = trilinear interpolation of channel ch of the network output
// (cell-centred coarse grid of level L) at the fine cell centre, divided by
// the feature scale and multiplied by the network's output scale (the RMS
// its training targets were divided by); 0 in cells outside the system
// (diag == 0)
template <typename V>
__global__ void prolong_trilinear_kernel(const float* __restrict__ out2, int ch, int X, int Y, int Z, int L,
                                         const double* __restrict__ scale, float out_scale,
                                         const double* __restrict__ diag, V* __restrict__ w, int ni, int nj, int nk) {
  const size_t n = (size_t)ni * nj * nk;
  const double s = *scale;
  const double inv_s = s > 0.0 ? (double)out_scale / s : 0.0;
  const float inv_b = 1.0f / (float)(1 << L);
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    if (!(diag[e] > 0.0)) {
      w[e] = V(0);
      continue;
    }
    int i, j, k;
    decode3(e, ni, nj, i, j, k);
    const float cx = fminf(fmaxf((i + 0.5f) * inv_b - 0.5f, 0.0f), (float)(X - 1));
    const float cy = fminf(fmaxf((j + 0.5f) * inv_b - 0.5f, 0.0f), (float)(Y - 1));
    const float cz = fminf(fmaxf((k + 0.5f) * inv_b - 0.5f, 0.0f), (float)(Z - 1));
    const int x0 = min((int)cx, X - 1), y0 = min((int)cy, Y - 1), z0 = min((int)cz, Z - 1);
    const int x1 = min(x0 + 1, X - 1), y1 = min(y0 + 1, Y - 1), z1 = min(z0 + 1, Z - 1);
    const float fx = cx - x0, fy = cy - y0, fz = cz - z0;
    auto at = [&](int x, int y, int z) { return out2[2 * (((size_t)z * Y + y) * X + x) + ch]; };
    const float c00 = at(x0, y0, z0) + fx * (at(x1, y0, z0) - at(x0, y0, z0));
    const float c10 = at(x0, y1, z0) + fx * (at(x1, y1, z0) - at(x0, y1, z0));
    const float c01 = at(x0, y0, z1) + fx * (at(x1, y0, z1) - at(x0, y0, z1));
    const float c11 = at(x0, y1, z1) + fx * (at(x1, y1, z1) - at(x0, y1, z1));
    const float c0 = c00 + fy * (c10 - c00), c1 = c01 + fy * (c11 - c01);
    w[e] = cvt<V>((typename Num<V>::Acc)((double)(c0 + fz * (c1 - c0)) * inv_s));
  }
}

// y += x
template <typename V>
__global__ void vec_add_kernel(V* __restrict__ y, const V* __restrict__ x, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = cvt<V>((typename Num<V>::Acc)((double)ldv(y + i) + (double)ldg(x + i)));
}

// y = A x for the 7-point operator stored as (diag, +x, +y, +z)
template <typename S, typename V>
__global__ void spmv_kernel(const V* __restrict__ x, V* __restrict__ y, const S* __restrict__ diag,
                            const S* __restrict__ xp, const S* __restrict__ yp, const S* __restrict__ zp, int ni,
                            int nj, int nk) {
  using A = typename Num<V>::Acc;
  const size_t n = (size_t)ni * nj * nk, sy = (size_t)ni, sz = (size_t)ni * nj;
  for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(g, ni, nj, i, j, k);
    A acc = A(0);
    if (k > 0) acc = acc + (A)ldg(zp + g - sz) * ldg(x + g - sz);
    if (j > 0) acc = acc + (A)ldg(yp + g - sy) * ldg(x + g - sy);
    if (i > 0) acc = acc + (A)ldg(xp + g - 1) * ldg(x + g - 1);
    acc = acc + (A)ldg(diag + g) * ldg(x + g);
    if (i < ni - 1) acc = acc + (A)ldg(xp + g) * ldg(x + g + 1);
    if (j < nj - 1) acc = acc + (A)ldg(yp + g) * ldg(x + g + sy);
    if (k < nk - 1) acc = acc + (A)ldg(zp + g) * ldg(x + g + sz);
    y[g] = cvt<V>(acc);
  }
}

// The Ritz step over W = [w0 .. w3] (unused vectors are all zero), Q = A W.
constexpr int kRitzVecs = 4;
constexpr int kRitzSums = kRitzVecs * (kRitzVecs + 1) / 2 + kRitzVecs;  // upper G, then W^T b
template <typename V>
struct RitzVecs {
  const V* w[kRitzVecs];
  const V* q[kRitzVecs];
  double gamma[kRitzVecs];
};

// FP64 block partials of G_ij = w_i.q_j (i <= j, row-major upper triangle)
// and g_i = w_i.b, written as partials[k * gridDim.x + block]
template <typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) ritz_dots_kernel(const RitzVecs<V> v, const V* __restrict__ b, size_t n,
                                                          double* partials) {
  __shared__ double sm[BLOCK / 32];
  double s[kRitzSums];
#pragma unroll
  for (int k = 0; k < kRitzSums; ++k) s[k] = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    double w[kRitzVecs], q[kRitzVecs];
#pragma unroll
    for (int a = 0; a < kRitzVecs; ++a) {
      w[a] = (double)ldg(v.w[a] + i);
      q[a] = (double)ldg(v.q[a] + i);
    }
    const double bb = (double)ldg(b + i);
    int k = 0;
#pragma unroll
    for (int a = 0; a < kRitzVecs; ++a)
#pragma unroll
      for (int c = a; c < kRitzVecs; ++c) s[k++] += w[a] * q[c];
#pragma unroll
    for (int a = 0; a < kRitzVecs; ++a) s[k++] += w[a] * bb;
  }
  for (int k = 0; k < kRitzSums; ++k) {
    const double t = block_sum<BLOCK>(s[k], sm);
    if (threadIdx.x == 0) partials[(size_t)k * gridDim.x + blockIdx.x] = t;
  }
}

// folds the partial rows in block order into out[kRitzSums] (one block)
template <int BLOCK>
__global__ void ritz_fold_kernel(const double* __restrict__ partials, int nb, double* __restrict__ out) {
  __shared__ double sm[BLOCK / 32];
  for (int k = 0; k < kRitzSums; ++k) {
    double v = 0.0;
    for (int q = threadIdx.x; q < nb; q += BLOCK) v += partials[(size_t)k * nb + q];
    v = block_sum<BLOCK>(v, sm);
    if (threadIdx.x == 0) out[k] = v;
  }
}

// x = sum gamma_i w_i, r = b - sum gamma_i q_i, partial |r|_inf (converged
// flag set against the tolerance by the last block)
template <typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) ritz_combine_kernel(const RitzVecs<V> v, const V* __restrict__ b,
                                                             V* __restrict__ x, V* __restrict__ r, size_t n,
                                                             double* partials, PcgScalars* st) {
  __shared__ double sm[BLOCK / 32];
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    double xv = 0.0, av = 0.0;
#pragma unroll
    for (int a = 0; a < kRitzVecs; ++a) {
      xv += v.gamma[a] * (double)ldg(v.w[a] + i);
      av += v.gamma[a] * (double)ldg(v.q[a] + i);
    }
    x[i] = cvt<V>((typename Num<V>::Acc)xv);
    const V rt = cvt<V>((typename Num<V>::Acc)((double)ldg(b + i) - av));
    r[i] = rt;
    m = fmax(m, fabs((double)ldv(&rt)));
  }
  const double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes, 0.0, gridDim.x);
}

// ---- the warm-start correction (residual mode): the previous pressure p
// and the network's correction e of its residual r0 = b - A p.

// r -= q (r0 = b - A p in place of r = b), its copy rv in the V-cycle's type
template <typename V>
__global__ void resid_sub_kernel(double* __restrict__ r, const double* __restrict__ q, V* __restrict__ rv, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = r[i] - q[i];
    r[i] = v;
    rv[i] = cvt<V>((typename Num<V>::Acc)v);
  }
}

// FP64 block partials of the 2 x 2 Ritz system over {p, e}: p.Ap, p.Ae,
// e.Ae, p.b, e.b, written as partials[k * gridDim.x + block]
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) ritz2_dots_kernel(const double* __restrict__ p, const double* __restrict__ ap,
                                                           const double* __restrict__ e, const double* __restrict__ ae,
                                                           const double* __restrict__ b, size_t n, double* partials) {
  __shared__ double sm[BLOCK / 32];
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    const double pv = __ldg(p + i), ev = __ldg(e + i), bv = __ldg(b + i), aev = __ldg(ae + i);
    s[0] += pv * __ldg(ap + i);
    s[1] += pv * aev;
    s[2] += ev * aev;
    s[3] += pv * bv;
    s[4] += ev * bv;
  }
  for (int k = 0; k < 5; ++k) {
    const double t = block_sum<BLOCK>(s[k], sm);
    if (threadIdx.x == 0) partials[(size_t)k * gridDim.x + blockIdx.x] = t;
  }
}

template <int BLOCK>
__global__ void ritz2_fold_kernel(const double* __restrict__ partials, int nb, double* __restrict__ out) {
  __shared__ double sm[BLOCK / 32];
  for (int k = 0; k < 5; ++k) {
    double v = 0.0;
    for (int q = threadIdx.x; q < nb; q += BLOCK) v += partials[(size_t)k * nb + q];
    v = block_sum<BLOCK>(v, sm);
    if (threadIdx.x == 0) out[k] = v;
  }
}

// x = g0 p + g1 e, r = b - g0 Ap - g1 Ae, rv = r in V, partial |r|_inf
// (g0, g1 = gam[0], gam[1], the device-side Ritz step's result)
// (the converged flag against the tolerance set by the last block)
template <typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) ritz2_combine_kernel(const double* __restrict__ p,
                                                              const double* __restrict__ ap,
                                                              const double* __restrict__ e,
                                                              const double* __restrict__ ae,
                                                              const double* __restrict__ b,
                                                              const double* __restrict__ gam,
                                                              double* __restrict__ x, double* __restrict__ r,
                                                              V* __restrict__ rv, size_t n, double* partials,
                                                              PcgScalars* st) {
  __shared__ double sm[BLOCK / 32];
  const double g0 = gam[0], g1 = gam[1];
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    x[i] = g0 * __ldg(p + i) + g1 * __ldg(e + i);
    const double rr = __ldg(b + i) - (g0 * __ldg(ap + i) + g1 * __ldg(ae + i));
    r[i] = rr;
    rv[i] = cvt<V>((typename Num<V>::Acc)rr);
    m = fmax(m, fabs(rr));
  }
  const double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes, 0.0, gridDim.x);
}

// x += alpha s; r_out = r_in - alpha q (r_in kept for the Polak-Ribiere beta)
template <typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) fcg_update_kernel(T* __restrict__ x, const T* __restrict__ r_in,
                                                          T* __restrict__ r_out, const T* __restrict__ s,
                                                          const T* __restrict__ q, size_t n, double* partials,
                                                          PcgScalars* st) {
  __shared__ double sm[BLOCK / 32];
  const double alpha = st->alpha;
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    const double xv = (double)ldv(x + i) + alpha * (double)ldg(s + i);
    const double rv = (double)ldg(r_in + i) - alpha * (double)ldg(q + i);
    const T rt = cvt<T>((typename Num<T>::Acc)rv);
    x[i] = cvt<T>((typename Num<T>::Acc)xv);
    r_out[i] = rt;
    m = fmax(m, fabs((double)ldv(&rt)));
  }
  const double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes, 0.0, gridDim.x);
}

}  // namespace vflip
