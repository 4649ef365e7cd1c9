// FP64 direct solve of the coarsest multigrid level (FP32 / mixed V-cycles).
//
// The reference relaxes its coarsest level with 200 red-black sweeps
// (AlgebraicMultigrid.h:160); the FP32 and mixed-precision contexts here
// may instead solve it exactly, in FP64, with a banded Cholesky factor
// built on the GPU each time the hierarchy is.  The coarsest operator is the
// 7-point Galerkin stencil of an ni x nj x nk grid; in lexicographic order
// its Cholesky factor L (A = L L^T) lives inside the band of half-width
// bw = ni*nj, stored by columns: Lc[c*(bw+1) + d] = L[c+d][c].
//
// Rows whose diagonal is zero (cells with no fluid at that level) are
// decoupled and solved as x = 0, as the red-black relaxation leaves them.
// A pivot that falls to 1e-12 of its diagonal (a singular block: a fluid
// region that no open boundary pins) clears the `ok` flag; the caller's
// red-black relaxation then runs instead (both kernels are launched, each
// returns at once when the flag says it is not the one wanted).
#pragma once
#include "common.cuh"

namespace vflip {

// A[c+d][c] of the symmetric 7-point operator given by its diagonal and its
// +x, +y, +z couplings; entries that touch a zero-diagonal row are 0.
__device__ __forceinline__ double band_entry(const double* diag, const double* xp, const double* yp,
                                             const double* zp, int ni, int nj, int nk, int c, int d) {
  const int n = ni * nj * nk;
  if (c >= n || c + d >= n) return 0.0;
  if (d == 0) return diag[c];
  if (diag[c] == 0.0 || diag[c + d] == 0.0) return 0.0;
  const int i = c % ni, j = (c / ni) % nj, k = c / (ni * nj);
  double v = 0.0;
  if (d == 1 && i < ni - 1) v += xp[c];
  if (d == ni && j < nj - 1) v += yp[c];
  if (d == ni * nj && k < nk - 1) v += zp[c];
  return v;
}

// One CTA.  Right-looking banded Cholesky with the bw+1 active columns in a
// shared-memory ring (column c in slot c mod (bw+1)): step k takes the pivot
// of column k, subtracts the rank-1 update of the scaled column k from
// columns k+1 .. k+bw, writes column k out and loads column k+bw+1 into its
// slot.  Two barriers per column.  FULL: the whole band (n columns of the
// original operator) is first staged in shared memory after the ring, so
// the loop's column loads and pivot tests read shared memory instead of
// waiting on a global load per column; the same arithmetic.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) coarse_chol_kernel(const double* __restrict__ diag,
                                                            const double* __restrict__ xp,
                                                            const double* __restrict__ yp,
                                                            const double* __restrict__ zp, int ni, int nj, int nk,
                                                            int bw, double* __restrict__ Lc,
                                                            double* __restrict__ rinv, int* __restrict__ ok_flag,
                                                            int full) {
  extern __shared__ double W[];
  __shared__ int ok;
  const int n = ni * nj * nk, B1 = bw + 1, tid = threadIdx.x;
  double* F = W + B1 * B1;  // FULL: column c of the band at F + c * B1
  if (full)
    for (int e = tid; e < n * B1; e += BLOCK) {
      const int c = e / B1, d = e - c * B1;
      F[e] = band_entry(diag, xp, yp, zp, ni, nj, nk, c, d);
    }
  for (int e = tid; e < B1 * B1; e += BLOCK) {
    const int c = e / B1, d = e - c * B1;
    W[e] = band_entry(diag, xp, yp, zp, ni, nj, nk, c, d);  // columns 0..bw in slots 0..bw
  }
  if (tid == 0) ok = 1;
  __syncthreads();
  int sk = 0;  // slot of column k
  for (int k = 0; k < n; ++k) {
    double* col = W + sk * B1;
    const double a = col[0], orig = full ? F[k * B1] : diag[k];
    const bool zero = orig == 0.0;
    const bool good = zero || (orig > 0.0 && a > 1e-12 * orig);
    const double l = (zero || !good) ? 1.0 : sqrt(a);
    const double il = 1.0 / l;
    // columns k+1 .. k+bw -= L[.][k] L[.][k]^T (pairs a >= b of offsets)
    if (!zero) {
      for (int e = tid; e < bw * bw; e += BLOCK) {
        const int oa = e / bw + 1, ob = e - (oa - 1) * bw + 1;
        if (ob > oa || k + oa >= n) continue;
        int s = sk + ob;
        if (s >= B1) s -= B1;
        W[s * B1 + (oa - ob)] -= (col[oa] * il) * (col[ob] * il);
      }
    }
    __syncthreads();
    // column k is final: write it out, then reuse its slot for column k+bw+1
    for (int d = tid; d < B1; d += BLOCK) {
      double v;
      if (d == 0) v = zero ? 1.0 : l;
      else v = (zero || k + d >= n) ? 0.0 : col[d] * il;
      Lc[(size_t)k * B1 + d] = v;
      col[d] = full ? (k + B1 < n ? F[(k + B1) * B1 + d] : 0.0) : band_entry(diag, xp, yp, zp, ni, nj, nk, k + B1, d);
    }
    if (tid == 0) {
      rinv[k] = zero ? 0.0 : il;
      if (!good) ok = 0;
    }
    __syncthreads();
    sk = sk + 1 == B1 ? 0 : sk + 1;
  }
  if (tid == 0) *ok_flag = ok;
}

// The band solve of coarse_chol_solve_kernel on y (shared memory, n
// values: b in, x out) by the whole CTA (nthreads >= 256 threads; the
// column sums of the backward pass use 8 threads per column of a 32-column
// block).  Every thread of the CTA calls it; it ends with a barrier.
__device__ __forceinline__ void chol_band_solve_block(double* y, int n, int bw, const double* Lc, const double* rinv,
                                                      int nthreads) {
  constexpr unsigned FULL = 0xffffffffu;
  const int B1 = bw + 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // ---- forward
  for (int kb = 0; kb < n; kb += 32) {
    const int nb = min(32, n - kb);
    if (warp == 0) {
      double yr = lane < nb ? y[kb + lane] : 0.0;
      for (int c = 0; c < nb; ++c) {
        const double lrc = (lane > c && lane < nb && lane - c <= bw) ? Lc[(size_t)(kb + c) * B1 + (lane - c)] : 0.0;
        const double yc = __shfl_sync(FULL, yr, c) * rinv[kb + c];
        if (lane == c) yr = yc;
        else if (lane > c) yr -= lrc * yc;
      }
      if (lane < nb) y[kb + lane] = yr;
    }
    __syncthreads();
    // rows below the block that the band reaches
    const int r0 = kb + nb, r1 = min(n, kb + nb + bw);
    for (int i = r0 + tid; i < r1; i += nthreads) {
      double s = y[i];
      for (int c = 0; c < nb; ++c) {
        const int d = i - (kb + c);
        if (d <= bw) s -= Lc[(size_t)(kb + c) * B1 + d] * y[kb + c];
      }
      y[i] = s;
    }
    __syncthreads();
  }
  // ---- backward
  const int last = ((n - 1) / 32) * 32;
  for (int kb = last; kb >= 0; kb -= 32) {
    const int nb = min(32, n - kb);
    // y[kb+r] -= sum over solved rows i >= kb+nb of L[i][kb+r] x[i]; eight
    // threads per column r, each over every eighth band offset
    {
      const int r = tid >> 3, part = tid & 7;
      double s = 0.0;
      if (r < nb) {
        const int c = kb + r;
        for (int d = kb + nb - c + part; d <= bw && c + d < n; d += 8) s += Lc[(size_t)c * B1 + d] * y[c + d];
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
        const double lcr = (lane < c && c - lane <= bw) ? Lc[(size_t)(kb + lane) * B1 + (c - lane)] : 0.0;
        const double xc = __shfl_sync(FULL, yr, c) * rinv[kb + c];
        if (lane == c) yr = xc;
        else if (lane < c) yr -= lcr * xc;
      }
      if (lane < nb) y[kb + lane] = yr;
    }
    __syncthreads();
  }
}

// One CTA: x = A^-1 b from the band factor, in FP64, blocked by 32 columns.
// With `staged`, the factor and the reciprocal pivots are first copied into
// shared memory (the whole solve then reads no global memory but b).
// Forward (L y = b): warp 0 solves each 32 x 32 diagonal block with
// shuffles, then all threads subtract the block's contribution from the
// next bw rows.  Backward (L^T x = y), blocks from the last: all threads
// first subtract the contributions of the rows already solved, then warp 0
// solves the block's transposed triangle.  With `dot_out`, also writes
// sum(x * b) (the PCG z.r when this level is the whole V-cycle).
// Returns at once unless *ok_flag is set.
template <typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) coarse_chol_solve_kernel(const V* __restrict__ b, V* __restrict__ x_out,
                                                                  int n, int bw, const double* Lc,
                                                                  const double* rinv,
                                                                  const int* __restrict__ ok_flag,
                                                                  double* __restrict__ dot_out, int staged) {
  if (*ok_flag == 0) return;
  extern __shared__ double y[];  // n values: y, then x in place; then the staged factor
  __shared__ double red[BLOCK / 32];
  constexpr unsigned FULL = 0xffffffffu;
  const int B1 = bw + 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < n; e += BLOCK) y[e] = (double)ldv(b + e);
  if (staged) {
    double* sL = y + n;
    for (int e = tid; e < n * B1; e += BLOCK) sL[e] = Lc[e];
    for (int e = tid; e < n; e += BLOCK) sL[n * B1 + e] = rinv[e];
    Lc = sL;
    rinv = sL + (size_t)n * B1;
  }
  __syncthreads();
  chol_band_solve_block(y, n, bw, Lc, rinv, BLOCK);
  double dot = 0.0;
  for (int e = tid; e < n; e += BLOCK) {
    const V o = cvt<V>(y[e]);
    x_out[e] = o;
    if (dot_out) dot += (double)ldv(&o) * (double)ldv(b + e);
  }
  if (dot_out) {
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(FULL, dot, o);
    if (lane == 0) red[warp] = dot;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int w = 0; w < BLOCK / 32; ++w) s += red[w];
      dot_out[0] = s;
    }
  }
}

}  // namespace vflip
