// PCG vector kernels and the on-device scalar recurrence of AMGPCGSolve
// (Smoke_Solver/AlgebraicMultigrid.h:189-301).
//
// The PCG scalars (rho, alpha, beta, the residual norm) live in device memory
// in FP64 for every precision mode; block partials of each reduction are
// combined in a fixed order by the last block to finish (threadfence +
// counter), so every reduction is deterministic run to run.
#pragma once
#include "common.cuh"

namespace vflip {

struct PcgScalars {
  double rho;        // z.r of the current iterate
  double rho_new;
  double rho_prev;   // z.r of the previous iterate (flexible PCG)
  double sz;         // s.(A s)
  double alpha;
  double beta;
  double res;        // |r|_inf
  double tol;        // tolerance_factor * |rhs|_inf
  double rhs_norm;   // |rhs|_inf
  int converged;     // res <= tol
  int bad_rho;       // rho == 0 or NaN
  int kernel_error;  // host copy of the smoother's timeout flag
  unsigned int done_blocks[5];  // last-block-done counters, one per reduction kind
};

enum ReduceKind { kReduceSZ = 0, kReduceRes = 1, kReduceRho = 2, kReduceRes0 = 3, kReduceFlex = 4 };

// Called by every thread of every block after thread 0 wrote the block's
// partial: the last block to arrive folds all partials in index order and
// updates the scalars.
template <int BLOCK>
__device__ __forceinline__ void finish_reduction(double* partials, int nblocks, PcgScalars* st, int kind,
                                                 double tol_factor, int launched_blocks) {
  __shared__ bool last;
  __shared__ double sm[BLOCK / 32];
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int ticket = atomicAdd(&st->done_blocks[kind], 1u);
    last = (ticket == (unsigned)launched_blocks - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // fold: each thread sums a fixed strided subset, then a fixed-order tree
  double v = 0.0;
  for (int q = threadIdx.x; q < nblocks; q += BLOCK) {
    double p = ((volatile double*)partials)[q];
    if (kind == kReduceRes || kind == kReduceRes0) v = fmax(v, p);
    else v += p;
  }
  double tot = (kind == kReduceRes || kind == kReduceRes0) ? block_absmax<BLOCK>(v, sm) : block_sum<BLOCK>(v, sm);
  if (threadIdx.x == 0) {
    st->done_blocks[kind] = 0;
    if (kind == kReduceSZ) {
      st->sz = tot;
      st->alpha = st->rho / tot;
    } else if (kind == kReduceRes) {
      st->res = tot;
      st->converged = (tot <= st->tol) ? 1 : 0;
    } else if (kind == kReduceRes0) {
      st->res = tot;
      st->rhs_norm = tot;
      st->tol = tol_factor * tot;
      st->converged = (tot == 0.0) ? 1 : 0;
    } else if (kind == kReduceFlex) {  // z_new . r_old: Polak-Ribiere beta of flexible PCG
      st->beta = (st->rho - tot) / st->rho_prev;
    } else {  // kReduceRho
      st->rho_new = tot;
      st->beta = tot / st->rho;  // unused after the first V-cycle (s = z there)
      st->rho_prev = st->rho;
      st->rho = tot;
      st->bad_rho = (tot == 0.0 || tot != tot) ? 1 : 0;
    }
  }
}

// Folds partials already written by another kernel (the fused dot of the
// last smoothing sweep); launched with a single block.
template <int BLOCK>
__global__ void fold_kernel(double* partials, int nblocks, PcgScalars* st, int kind, double tol_factor) {
  // a single block performs the whole fold
  finish_reduction<BLOCK>(partials, nblocks, st, kind, tol_factor, 1);
}

// r = rhs (converted to the vector type), x = 0, partial |rhs|_inf.
template <typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) pcg_init_kernel(const double* __restrict__ rhs, T* __restrict__ r,
                                                        T* __restrict__ x, size_t n, double* partials,
                                                        PcgScalars* st, double tol_factor) {
  __shared__ double sm[BLOCK / 32];
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    double v = rhs[i];
    r[i] = cvt<T>((typename Num<T>::Acc)v);
    x[i] = cvt<T>((typename Num<T>::Acc)0);
    m = fmax(m, fabs(v));
  }
  double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes0, tol_factor, gridDim.x);
}

// s_new = first ? z : z + beta*s_old   (AlgebraicMultigrid.h:254, 284)
// q = A s_new                           (multiply, sparse_matrix.h:356-362)
// partial s_new.q                        (AlgebraicMultigrid.h:259)
// One thread per cell of a (32 x 8) x-y tile, marching k.  The neighbours'
// s_new are recomputed from z and s_old, so s_old is never overwritten.
// TZ: the preconditioned residual's type (the V-cycle's vectors), which
// may be narrower than the PCG vectors' T.
// TO: storage of the off-diagonal couplings (T, or float where the FP64
// operator's couplings are exactly FP32 values: products and sums then run
// in T on the same values).
template <typename T, bool FIRST, int BLOCK, typename TZ = T, typename TO = T>
__global__ void __launch_bounds__(BLOCK) pcg_spmv_dot_kernel(const TZ* __restrict__ z, const T* __restrict__ s_old,
                                                            T* __restrict__ s_new, T* __restrict__ q,
                                                            const T* __restrict__ diag, const TO* __restrict__ xp,
                                                            const TO* __restrict__ yp, const TO* __restrict__ zp,
                                                            int ni, int nj, int nk, int kz, double* partials,
                                                            PcgScalars* st) {
  using A = typename Num<T>::Acc;
  __shared__ double sm[BLOCK / 32];
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  const int j = blockIdx.y * (BLOCK / 32) + (threadIdx.x >> 5);
  const int kb = blockIdx.z * kz, ke = min(kb + kz, nk);
  const size_t sy = (size_t)ni, szs = (size_t)ni * nj;
  const double beta = FIRST ? 0.0 : st->beta;
  double dot = 0.0;
  if (i < ni && j < nj) {
    for (int k = kb; k < ke; ++k) {
      size_t g = lin3(i, j, k, ni, nj);
      auto sv = [&](size_t gg) -> A {
        if (FIRST) return A(ldg(z + gg));
        T t = cvt<T>((A)((double)ldg(z + gg) + beta * (double)ldg(s_old + gg)));
        return ldv(&t);
      };
      A sc = sv(g);
      A acc = A(0);
      if (k > 0) acc = acc + ldg(zp + g - szs) * sv(g - szs);
      if (j > 0) acc = acc + ldg(yp + g - sy) * sv(g - sy);
      if (i > 0) acc = acc + ldg(xp + g - 1) * sv(g - 1);
      acc = acc + ldg(diag + g) * sc;
      if (i < ni - 1) acc = acc + ldg(xp + g) * sv(g + 1);
      if (j < nj - 1) acc = acc + ldg(yp + g) * sv(g + sy);
      if (k < nk - 1) acc = acc + ldg(zp + g) * sv(g + szs);
      if (s_new) s_new[g] = cvt<T>(sc);
      T qq = cvt<T>(acc);
      q[g] = qq;
      dot += (double)sc * (double)ldv(&qq);
    }
  }
  double bs = block_sum<BLOCK>(dot, sm);
  int nb = gridDim.x * gridDim.y * gridDim.z;
  int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (threadIdx.x == 0) partials[bid] = bs;
  finish_reduction<BLOCK>(partials, nb, st, kReduceSZ, 0.0, nb);
}

// The same step as pcg_spmv_dot_kernel for grids whose rows are whole
// quads (ni % 4 == 0): one thread per quad of 4 consecutive cells, a block
// per (TY rows + one halo row either side) x (a range of planes), marching k.
// Each cell's s_new is formed once per block: z-neighbours ride in
// registers (three planes), x- and y-neighbours and the -y couplings come
// from a three-plane shared-memory ring that every thread writes once per
// plane, so one barrier per plane suffices.  The halo rows only form s and
// yp.  q of plane k-1 is computed in the step that forms plane k.  Each
// cell's q sums its terms in pcg_spmv_dot_kernel's order (-z, -y, -x, diag,
// +x, +y, +z) with the same roundings, so q and s_new are bitwise those of
// that kernel; the partial dots are grouped differently (deterministic).
template <typename T>
struct alignas(4 * sizeof(T)) Quad {
  T v[4];
};

template <typename T>
__device__ __forceinline__ Quad<T> ldq(const T* p) {
  return *reinterpret_cast<const Quad<T>*>(p);
}

template <typename T, bool FIRST, typename TZ = T, typename TO = T>
__global__ void __launch_bounds__(1024) pcg_spmv_dot_plane_kernel(
    const TZ* __restrict__ z, const T* __restrict__ s_old, T* __restrict__ s_new, T* __restrict__ q,
    const T* __restrict__ diag, const TO* __restrict__ xp, const TO* __restrict__ yp, const TO* __restrict__ zp,
    int ni, int nj, int nk, int ty, int kz, double* partials, PcgScalars* st) {
  using A = typename Num<T>::Acc;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int qx = threadIdx.x, ry = threadIdx.y, nq = blockDim.x, rows = blockDim.y;  // rows = ty + 2
  Quad<T>* sbuf = reinterpret_cast<Quad<T>*>(smem_raw);                      // [3][rows][nq]
  Quad<TO>* ybuf = reinterpret_cast<Quad<TO>*>(sbuf + 3 * rows * nq);        // [3][rows][nq]
  __shared__ double red[32];
  const int j = blockIdx.x * ty - 1 + ry;
  const bool in_row = j >= 0 && j < nj;
  const bool interior = ry >= 1 && ry <= ty && in_row;
  const int kb = blockIdx.y * kz, ke = min(kb + kz, nk);
  const size_t sy = (size_t)ni, szs = (size_t)ni * nj;
  const int i0 = 4 * qx;
  const double beta = FIRST ? 0.0 : st->beta;
  Quad<T> sm{}, sc{}, sp{};  // s of planes k-1, k, k+1 (relative to the q plane)
  Quad<TO> zprev{};          // zp of the plane below the q plane
  double dot = 0.0;
  for (int kk = kb - 1; kk <= ke; ++kk) {
    // s_new of plane kk on this thread's row
    Quad<T> snew{};
    Quad<TO> ypk{};
    if (in_row && kk >= 0 && kk < nk) {
      const size_t g = (size_t)i0 + sy * j + szs * kk;
      const Quad<TZ> zq = ldq(z + g);
      if (FIRST) {
#pragma unroll
        for (int c = 0; c < 4; ++c) snew.v[c] = cvt<T>(A(ldv(&zq.v[c])));
      } else {
        const Quad<T> so = ldq(s_old + g);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          snew.v[c] = cvt<T>((A)((double)ldv(&zq.v[c]) + beta * (double)ldv(&so.v[c])));
      }
      if (ry <= ty) ypk = ldq(yp + g);
    }
    const int bw = (kk + 3) % 3;  // kk >= -1
    sbuf[(bw * rows + ry) * nq + qx] = snew;
    ybuf[(bw * rows + ry) * nq + qx] = ypk;
    sm = sc;
    sc = sp;
    sp = snew;
    __syncthreads();
    const int k = kk - 1;  // the q plane
    if (interior && k >= kb && k < ke) {
      const size_t g = (size_t)i0 + sy * j + szs * k;
      const int br = (k + 3) % 3;
      const Quad<T> dq = ldq(diag + g);
      const Quad<TO> xq = ldq(xp + g), zq = ldq(zp + g);
      const Quad<TO> yq = ybuf[(br * rows + ry) * nq + qx];
      const Quad<T> sdn = sbuf[(br * rows + ry - 1) * nq + qx];
      const Quad<TO> ydn = ybuf[(br * rows + ry - 1) * nq + qx];
      const Quad<T> sup = sbuf[(br * rows + ry + 1) * nq + qx];
      // x-neighbours: the left and right cells of each cell of the quad, and
      // the -x coupling (xp of the cell to the left)
      A sleft[4], sright[4], xleft[4];
      sleft[0] = qx > 0 ? ldv(&sbuf[(br * rows + ry) * nq + qx - 1].v[3]) : A(0);
      xleft[0] = qx > 0 ? ldg(xp + g - 1) : A(0);
      sright[3] = qx + 1 < nq ? ldv(&sbuf[(br * rows + ry) * nq + qx + 1].v[0]) : A(0);
#pragma unroll
      for (int c = 1; c < 4; ++c) {
        sleft[c] = ldv(&sc.v[c - 1]);
        xleft[c] = ldv(&xq.v[c - 1]);
        sright[c - 1] = ldv(&sc.v[c]);
      }
      Quad<T> qo;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int i = i0 + c;
        A acc = A(0);
        if (k > 0) acc = acc + ldv(&zprev.v[c]) * ldv(&sm.v[c]);
        if (j > 0) acc = acc + ldv(&ydn.v[c]) * ldv(&sdn.v[c]);
        if (i > 0) acc = acc + xleft[c] * sleft[c];
        acc = acc + ldv(&dq.v[c]) * ldv(&sc.v[c]);
        if (i < ni - 1) acc = acc + ldv(&xq.v[c]) * sright[c];
        if (j < nj - 1) acc = acc + ldv(&yq.v[c]) * ldv(&sup.v[c]);
        if (k < nk - 1) acc = acc + ldv(&zq.v[c]) * ldv(&sp.v[c]);
        qo.v[c] = cvt<T>(acc);
        dot += (double)ldv(&sc.v[c]) * (double)ldv(&qo.v[c]);
      }
      *reinterpret_cast<Quad<T>*>(q + g) = qo;
      if (s_new) *reinterpret_cast<Quad<T>*>(s_new + g) = sc;
      zprev = zq;
    } else if (interior && k == kb - 1 && k >= 0) {
      // the plane below the first q plane: only its zp is carried
      zprev = ldq(zp + (size_t)i0 + sy * j + szs * k);
    }
  }
  // block sum in a fixed order: warp trees, then warps in index order
  const int tid = qx + nq * ry, nthreads = nq * rows;
  for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
  if ((tid & 31) == 0) red[tid >> 5] = dot;
  __syncthreads();
  const int bid = blockIdx.x + gridDim.x * blockIdx.y, nb = gridDim.x * gridDim.y;
  if (tid == 0) {
    double b = 0.0;
    for (int w = 0; w < (nthreads + 31) / 32; ++w) b += red[w];
    partials[bid] = b;
  }
  // finish_reduction's fold needs a 1-D view of the block: thread 0 arrives
  // for the block, the last block's threads fold
  __shared__ bool last;
  if (tid == 0) {
    __threadfence();
    const unsigned int ticket = atomicAdd(&st->done_blocks[kReduceSZ], 1u);
    last = (ticket == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (int p = tid; p < nb; p += nthreads) v += ((volatile double*)partials)[p];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    double tot = 0.0;
    for (int w = 0; w < (nthreads + 31) / 32; ++w) tot += red[w];
    st->done_blocks[kReduceSZ] = 0;
    st->sz = tot;
    st->alpha = st->rho / tot;
  }
}

// x += alpha s, r -= alpha q, partial |r|_inf  (AlgebraicMultigrid.h:259-262)
template <typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) pcg_update_kernel(T* __restrict__ x, T* __restrict__ r,
                                                          const T* __restrict__ s, const T* __restrict__ q, size_t n,
                                                          double* partials, PcgScalars* st) {
  __shared__ double sm[BLOCK / 32];
  const double alpha = st->alpha;
  const double nalpha = -alpha;
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    double xv = (double)ldv(x + i) + alpha * (double)ldg(s + i);
    double rv = (double)ldv(r + i) + nalpha * (double)ldg(q + i);
    T rt = cvt<T>((typename Num<T>::Acc)rv);
    x[i] = cvt<T>((typename Num<T>::Acc)xv);
    r[i] = rt;
    m = fmax(m, fabs((double)ldv(&rt)));
  }
  double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes, 0.0, gridDim.x);
}

// FP64 outer loop around a narrower V-cycle (vectors of type V):
// r = rhs, its copy rv in V for the V-cycle, x = 0, partial |rhs|_inf.
template <typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) pcg_init_outer_kernel(const double* __restrict__ rhs, double* __restrict__ r,
                                                              V* __restrict__ rv, double* __restrict__ x, size_t n,
                                                              double* partials, PcgScalars* st, double tol_factor) {
  __shared__ double sm[BLOCK / 32];
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    const double v = rhs[i];
    r[i] = v;
    rv[i] = cvt<V>((typename Num<V>::Acc)v);
    x[i] = 0.0;
    m = fmax(m, fabs(v));
  }
  double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes0, tol_factor, gridDim.x);
}

// x += alpha s, r -= alpha q in FP64, the V-cycle's copy rv = r, partial |r|_inf
template <typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) pcg_update_outer_kernel(double* __restrict__ x, double* __restrict__ r,
                                                                V* __restrict__ rv, const double* __restrict__ s,
                                                                const double* __restrict__ q, size_t n,
                                                                double* partials, PcgScalars* st) {
  __shared__ double sm[BLOCK / 32];
  const double alpha = st->alpha;
  const double nalpha = -alpha;
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK) {
    const double xv = x[i] + alpha * __ldg(s + i);
    const double rr = r[i] + nalpha * __ldg(q + i);
    x[i] = xv;
    r[i] = rr;
    rv[i] = cvt<V>((typename Num<V>::Acc)rr);
    m = fmax(m, fabs(rr));
  }
  double bm = block_absmax<BLOCK>(m, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bm;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kReduceRes, 0.0, gridDim.x);
}

// Plain z.r when the V-cycle could not fuse it (single-level hierarchies
// produce it inside the coarsest kernel instead).
template <typename T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) dot_kernel(const T* __restrict__ a, const T* __restrict__ b, size_t n,
                                                   double* partials, PcgScalars* st, int kind) {
  __shared__ double sm[BLOCK / 32];
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK)
    s += (double)ldg(a + i) * (double)ldg(b + i);
  double bs = block_sum<BLOCK>(s, sm);
  if (threadIdx.x == 0) partials[blockIdx.x] = bs;
  finish_reduction<BLOCK>(partials, gridDim.x, st, kind, 0.0, gridDim.x);
}

// ---- graph-resident PCG (batched solves): the loop runs as a CUDA graph
// while-node whose condition a kernel sets from the device-side scalars.

// after pcg_init: rho = 1 so the first beta only scales s = 0
__global__ void pcg_loop_init_kernel(PcgScalars* st, int* it, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    st->rho = 1.0;
    st->beta = 0.0;
    *it = 0;
    cudaGraphSetConditional(h, st->converged ? 0u : 1u);
  }
}

// s = z + beta s in place (the direction update of AlgebraicMultigrid.h:284)
template <typename T, typename TZ = T>
__global__ void pcg_direction_kernel(const TZ* __restrict__ z, T* __restrict__ s, size_t n, const PcgScalars* st) {
  using A = typename Num<T>::Acc;
  const double beta = st->beta;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    s[i] = cvt<T>((A)((double)ldg(z + i) + beta * (double)ldv(s + i)));
}

// one iteration done: continue while not converged, rho valid, below maxit
__global__ void pcg_loop_cond_kernel(const PcgScalars* st, int* it, int maxit, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const int k = ++*it;
    const bool go = !st->converged && !st->bad_rho && k < maxit && st->res == st->res;
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

template <typename T, int BLOCK>
__global__ void to_double_kernel(const T* __restrict__ src, double* __restrict__ dst, size_t n) {
  for (size_t i = (size_t)blockIdx.x * BLOCK + threadIdx.x; i < n; i += (size_t)gridDim.x * BLOCK)
    dst[i] = (double)ldg(src + i);
}

}  // namespace vflip
