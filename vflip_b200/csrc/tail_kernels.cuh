// The small end of the V-cycle (amgVCycle, AlgebraicMultigrid.h:130-176) in
// ONE CTA: every level from the first one of at most kTailMaxCells cells
// down to the coarsest, held in shared memory.
//
// Below 16^3 cells a level's sweep is a few thousand cells: launched as its
// own kernel it costs the launch and the plane pipeline's fill, several
// microseconds for almost no work, and a V-cycle has nine such launches per
// level.  Here a level's pre-smoothing, restriction, the coarsest solve and
// the post-smoothing with the prolongation are colour passes over shared
// memory separated by CTA barriers.
//
// The values are those of the launched kernels bit for bit: the same
// red-black order (colour 1, then colour 0), the same row-sum order and
// fused multiply-adds (gs_madd, skipping the terms of neighbours outside the
// level, which the launched kernels add as +-0), the same division, the
// residual_restrict_kernel arithmetic for the restriction (-fmad=false:
// every product and sum rounded as written), x + P x_c (injection) before
// the first post-sweep, and the coarsest level solved by the same FP64 band
// Cholesky steps (chol_band_solve_block) or, without a valid factor, by the
// coarsest_rbgs_kernel sweeps from zero.
#pragma once
#include "coarse_direct.cuh"
#include "common.cuh"

namespace vflip {

constexpr int kTailThreads = 1024;
constexpr int kTailMaxLevels = 8;
constexpr int kTailMaxCells = 4096;

template <typename S>
struct TailLevel {
  int ni, nj, nk;
  const S* diag;
  const S* xp;
  const S* yp;
  const S* zp;
};

template <typename S, typename V>
struct TailArgs {
  int nlev;  // levels in the tail (lv[nlev-1] is the coarsest), >= 1
  TailLevel<S> lv[kTailMaxLevels];
  const V* b;  // right-hand side of the tail's first level (global)
  V* x;        // its result (global)
  int pre, post, coarse_sweeps;
  int direct, bw;  // coarsest level: the FP64 band-Cholesky factor, used when direct and *ok
  const double* L;
  const double* rinv;
  const int* ok;
};

// shared-memory floats of one level: x, b, diag, xp, yp, zp, then one
// mask byte per cell (bits 0-5: which of the six neighbours exist, in the
// row-sum order -z, -y, -x, +x, +y, +z; bit 6: the cell's colour), packed
// four to a float slot
__host__ __device__ inline size_t tail_level_floats(int n) { return 6 * (size_t)n + ((size_t)n + 3) / 4; }

// One red-black sweep in place on a level held in shared memory; the masks
// spare the index arithmetic (sy = ni, sz = ni * nj).
__device__ __forceinline__ void tail_sweep(float* xs, const float* bs, const float* ds, const float* xps,
                                           const float* yps, const float* zps, const unsigned char* mk, int n,
                                           int sy, int sz) {
  for (int parity = 1; parity >= 0; --parity) {
    for (int e = threadIdx.x; e < n; e += kTailThreads) {
      const int f = mk[e];
      if ((f >> 6) != parity) continue;
      float sum = 0.0f;
      if (f & 1) sum = gs_madd(sum, zps[e - sz], xs[e - sz]);
      if (f & 2) sum = gs_madd(sum, yps[e - sy], xs[e - sy]);
      if (f & 4) sum = gs_madd(sum, xps[e - 1], xs[e - 1]);
      if (f & 8) sum = gs_madd(sum, xps[e], xs[e + 1]);
      if (f & 16) sum = gs_madd(sum, yps[e], xs[e + sy]);
      if (f & 32) sum = gs_madd(sum, zps[e], xs[e + sz]);
      const float d = ds[e];
      xs[e] = (d != 0.0f) ? gs_div(bs[e] - sum, d) : 0.0f;
    }
    __syncthreads();
  }
}

template <typename S, typename V>
__global__ void __launch_bounds__(kTailThreads) tail_vcycle_kernel(const TailArgs<S, V> a) {
  extern __shared__ __align__(16) float tsm[];
  const int tid = threadIdx.x, L = a.nlev;
  // shared-memory layout: per level x, b, diag, xp, yp, zp; then the FP64
  // vector of the coarsest direct solve
  float* base[kTailMaxLevels];
  size_t off = 0;
  for (int l = 0; l < L; ++l) {
    base[l] = tsm + off;
    off += tail_level_floats(a.lv[l].ni * a.lv[l].nj * a.lv[l].nk);
  }
  double* ydir = reinterpret_cast<double*>(tsm + ((off + 1) & ~(size_t)1));
  auto X = [&](int l) { return base[l]; };
  auto cnt = [&](int l) { return a.lv[l].ni * a.lv[l].nj * a.lv[l].nk; };
  for (int l = 0; l < L; ++l) {
    const int n = cnt(l);
    float* p = base[l];
    const TailLevel<S>& v = a.lv[l];
    unsigned char* mk = reinterpret_cast<unsigned char*>(p + 6 * n);
    const int ni = v.ni, nj = v.nj, nk = v.nk;
    for (int e = tid; e < n; e += kTailThreads) {
      p[e] = 0.0f;
      p[n + e] = l == 0 ? (float)ldv(a.b + e) : 0.0f;
      p[2 * n + e] = (float)ldv(v.diag + e);
      p[3 * n + e] = (float)ldv(v.xp + e);
      p[4 * n + e] = (float)ldv(v.yp + e);
      p[5 * n + e] = (float)ldv(v.zp + e);
      const int i = e % ni, j = (e / ni) % nj, k = e / (ni * nj);
      mk[e] = (unsigned char)((k > 0) | ((j > 0) << 1) | ((i > 0) << 2) | ((i < ni - 1) << 3) |
                              ((j < nj - 1) << 4) | ((k < nk - 1) << 5) | (((i + j + k) & 1) << 6));
    }
  }
  __syncthreads();
  auto sweep_level = [&](int l) {
    const int n = cnt(l);
    float* p = base[l];
    tail_sweep(p, p + n, p + 2 * n, p + 3 * n, p + 4 * n, p + 5 * n, reinterpret_cast<const unsigned char*>(p + 6 * n),
               n, a.lv[l].ni, a.lv[l].ni * a.lv[l].nj);
  };
  // ---- down: x = 0, pre-sweeps, b_{l+1} = R (b - A x)
  for (int l = 0; l + 1 < L; ++l) {
    for (int s = 0; s < a.pre; ++s) sweep_level(l);
    const int ni = a.lv[l].ni, nj = a.lv[l].nj, nk = a.lv[l].nk, n = cnt(l), sy = ni, sz = ni * nj;
    const float* xs = X(l);
    const float *bs = xs + n, *ds = xs + 2 * n, *xps = xs + 3 * n, *yps = xs + 4 * n, *zps = xs + 5 * n;
    const int cni = a.lv[l + 1].ni, cnj = a.lv[l + 1].nj, cn = cnt(l + 1);
    float* bc = X(l + 1) + cn;
    for (int c = tid; c < cn; c += kTailThreads) {
      const int I = c % cni, J = (c / cni) % cnj, K = c / (cni * cnj);
      float s = 0.0f;
      for (int kk = 0; kk <= 1; ++kk)
        for (int jj = 0; jj <= 1; ++jj)
          for (int ii = 0; ii <= 1; ++ii) {
            const int i = 2 * I + ii, j = 2 * J + jj, k = 2 * K + kk;
            if (i >= ni || j >= nj || k >= nk) continue;
            const int g = (k * nj + j) * ni + i;
            float r = bs[g];
            if (k > 0) r = r - zps[g - sz] * xs[g - sz];
            if (j > 0) r = r - yps[g - sy] * xs[g - sy];
            if (i > 0) r = r - xps[g - 1] * xs[g - 1];
            r = r - ds[g] * xs[g];
            if (i < ni - 1) r = r - xps[g] * xs[g + 1];
            if (j < nj - 1) r = r - yps[g] * xs[g + sy];
            if (k < nk - 1) r = r - zps[g] * xs[g + sz];
            s = s + 0.125f * r;
          }
      bc[c] = s;
    }
    __syncthreads();
  }
  // ---- the coarsest level
  {
    const int l = L - 1, n = cnt(l);
    float* p = base[l];
    if (a.direct && *a.ok != 0) {
      for (int e = tid; e < n; e += kTailThreads) ydir[e] = (double)p[n + e];
      __syncthreads();
      chol_band_solve_block(ydir, n, a.bw, a.L, a.rinv, kTailThreads);
      for (int e = tid; e < n; e += kTailThreads) p[e] = (float)ydir[e];
      __syncthreads();
    } else {
      for (int s = 0; s < a.coarse_sweeps; ++s) sweep_level(l);
    }
  }
  // ---- up: x += P x_c (injection), post-sweeps
  for (int l = L - 2; l >= 0; --l) {
    const int ni = a.lv[l].ni, nj = a.lv[l].nj, n = cnt(l);
    const int cni = a.lv[l + 1].ni, cnj = a.lv[l + 1].nj;
    float* xs = X(l);
    const float* xc = X(l + 1);
    for (int e = tid; e < n; e += kTailThreads) {
      const int i = e % ni, j = (e / ni) % nj, k = e / (ni * nj);
      xs[e] = xs[e] + xc[((k >> 1) * cnj + (j >> 1)) * cni + (i >> 1)];
    }
    __syncthreads();
    for (int s = 0; s < a.post; ++s) sweep_level(l);
  }
  const int n0 = cnt(0);
  for (int e = tid; e < n0; e += kTailThreads) a.x[e] = cvt<V>(X(0)[e]);
}

}  // namespace vflip
