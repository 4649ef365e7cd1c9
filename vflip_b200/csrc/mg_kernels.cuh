// Multigrid kernels: Galerkin coarsening, fused red-black Gauss-Seidel
// sweeps, residual+restriction, coarsest-level solve.
//
// All of them reproduce the arithmetic of the reference's CSR routines in
// the order the reference performs it, so the FP64 instantiation is
// bit-identical to the reference V-cycle (Smoke_Solver/AlgebraicMultigrid.h
// and GeometricLevelGen.*):
//   * a row sum walks the CSR columns in ascending order: -z, -y, -x,
//     (diag), +x, +y, +z;
//   * red-black GS updates colour (i+j+k) odd, then even (AlgebraicMultigrid.h:39,74);
//   * restriction adds 0.125*r over the children in ascending fine index,
//     prolongation adds the parent's value (injection).
#pragma once
#include "common.cuh"

namespace vflip {

// ---------------------------------------------------------------------------
// Galerkin coarsening, A_c = 0.5 R A P with R = 1/8 over the 2x2x2 children
// and P = injection (GeometricLevelGen.cpp:41-66, GeometricLevelGen.h:60-68,
// sparse_matrix.h:370-405).  Computed in FP64 on the stored half (diag, +x,
// +y, +z) of the symmetric operator.  0.5*0.125 = 0.0625 is a power of two,
// so scaling each child's partial row sum by it reproduces the two SpGEMMs
// term for term.  One thread per coarse cell.
__global__ void galerkin_coarsen_kernel(const double* __restrict__ fd, const double* __restrict__ fxp,
                                        const double* __restrict__ fyp, const double* __restrict__ fzp,
                                        double* __restrict__ cd, double* __restrict__ cxp,
                                        double* __restrict__ cyp, double* __restrict__ czp, int ni, int nj,
                                        int nk, int cni, int cnj, int cnk) {
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  int J = blockIdx.y * blockDim.y + threadIdx.y;
  int K = blockIdx.z;
  if (I >= cni || J >= cnj || K >= cnk) return;
  const size_t sx = 1, sy = (size_t)ni, sz = (size_t)ni * nj;
  double aD = 0, aX = 0, aY = 0, aZ = 0;
  bool hD = false, hX = false, hY = false, hZ = false;
#pragma unroll
  for (int kk = 0; kk <= 1; ++kk)
#pragma unroll
    for (int jj = 0; jj <= 1; ++jj)
#pragma unroll
      for (int ii = 0; ii <= 1; ++ii) {
        int fi = 2 * I + ii, fj = 2 * J + jj, fk = 2 * K + kk;
        if (fi >= ni || fj >= nj || fk >= nk) continue;
        size_t c = lin3(fi, fj, fk, ni, nj);
        // temp(c, parent): the child's row entries whose column has parent I,
        // summed in column order
        double t = 0;
        bool th = false;
        auto add = [&](double v) {
          if (th) t = __dadd_rn(t, v);
          else { t = v; th = true; }
        };
        if (kk == 1) add(fzp[c - sz]);
        if (jj == 1) add(fyp[c - sy]);
        if (ii == 1) add(fxp[c - sx]);
        add(fd[c]);
        if (ii == 0 && fi + 1 < ni) add(fxp[c]);
        if (jj == 0 && fj + 1 < nj) add(fyp[c]);
        if (kk == 0 && fk + 1 < nk) add(fzp[c]);
        double v = __dmul_rn(0.0625, t);
        if (hD) aD = __dadd_rn(aD, v); else { aD = v; hD = true; }
        if (ii == 1 && fi + 1 < ni) {
          double w = __dmul_rn(0.0625, fxp[c]);
          if (hX) aX = __dadd_rn(aX, w); else { aX = w; hX = true; }
        }
        if (jj == 1 && fj + 1 < nj) {
          double w = __dmul_rn(0.0625, fyp[c]);
          if (hY) aY = __dadd_rn(aY, w); else { aY = w; hY = true; }
        }
        if (kk == 1 && fk + 1 < nk) {
          double w = __dmul_rn(0.0625, fzp[c]);
          if (hZ) aZ = __dadd_rn(aZ, w); else { aZ = w; hZ = true; }
        }
      }
  size_t o = lin3(I, J, K, cni, cnj);
  cd[o] = aD;
  cxp[o] = aX;
  cyp[o] = aY;
  czp[o] = aZ;
}

template <typename T>
__global__ void convert_kernel(const double* __restrict__ src, T* __restrict__ dst, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) dst[i] = cvt<T>((typename Num<T>::Acc)src[i]);
}

// ---------------------------------------------------------------------------
// One full red-black Gauss-Seidel sweep (both colours), fused, out of place.
//
// In a red-black sweep the red update reads only black values and the black
// update reads only the new red values, so a sweep is a pure function of the
// incoming black values and b.  Each CTA owns full x-rows [j0, j0+tyo) of a
// z-chunk [k0, k0+kz) and marches k upward with a 4-plane rolling window in
// shared memory:
//   step p:  stage x_in plane p+1 (rows j0-2 .. j0+tyo+1)
//            red   update of plane p   on rows j0-1 .. j0+tyo  (one-row ring)
//            black update of plane p-1 on rows j0 .. j0+tyo-1
//            store plane p-1
// The ring rows and the planes k0-1 and k0+kz are recomputed redundantly by
// the neighbouring CTAs, so no CTA ever reads a value another CTA writes and
// x_in/x_out must be different buffers.
//
// Variants (compile-time):
//   ZERO_X  - the incoming x is zero (first pre-smoothing sweep of a level,
//             amgVCycle zero-fills x, AlgebraicMultigrid.h:145-152, 185-186);
//   PROLONG - the incoming x is x_in + P x_coarse (prolongation fused into the
//             first post-smoothing sweep, AlgebraicMultigrid.h:118-129,161-165);
//   DOT     - also accumulate sum(x_out * b) over the CTA's cells (the PCG
//             rho = dot(z, r) at the fine level, AlgebraicMultigrid.h:282).
template <typename S, typename V>
struct SweepArgs {
  const V* x_in;
  V* x_out;
  const V* b;
  const S* diag;
  const S* xp;
  const S* yp;
  const S* zp;
  const V* xc;  // coarse x (PROLONG)
  int ni, nj, nk;
  int cni, cnj;
  int tyo, kz;
  int plane_stride;  // elements per staged plane (>= (tyo+4)*ni)
  double* dot_partial;
};

template <typename S, typename V, bool ZERO_X, bool PROLONG, bool DOT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) rbgs_sweep_kernel(SweepArgs<S, V> a) {
  using A = typename Num<V>::Acc;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* xs = reinterpret_cast<A*>(smem_raw);
  __shared__ double red_smem[BLOCK / 32];

  const int ni = a.ni, nj = a.nj, nk = a.nk;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const int j0 = blockIdx.x * a.tyo;
  const int k0 = blockIdx.y * a.kz;
  const int kend = min(k0 + a.kz, nk);
  const int jout1 = min(j0 + a.tyo, nj);
  const int jr0 = max(j0 - 2, 0);                  // first staged row
  const int jr1 = min(j0 + a.tyo + 2, nj);         // one past the last staged row
  const int jred0 = max(j0 - 1, 0), jred1 = min(j0 + a.tyo + 1, nj);
  const int rows = jr1 - jr0;
  const int pls = a.plane_stride;
  auto X = [&](int p) -> A* { return xs + (size_t)(p & 3) * pls; };

  auto stage = [&](int q) {
    if (q < 0 || q >= nk) return;
    A* dst = X(q);
    const int cnt = rows * ni;
    const size_t base = (size_t)q * sz + (size_t)jr0 * sy;
    for (int e = threadIdx.x; e < cnt; e += BLOCK) {
      A v;
      if (ZERO_X) {
        v = A(0);
      } else {
        v = ldg(a.x_in + base + e);
        if (PROLONG) {
          int i = e % ni, j = jr0 + e / ni;
          v = v + ldg(a.xc + lin3(i >> 1, j >> 1, q >> 1, a.cni, a.cnj));
        }
      }
      dst[e] = v;
    }
  };

  // relax every cell of colour `parity` ((i+j+p)&1) on plane p, rows [r0, r1)
  auto relax = [&](int p, int r0, int r1, int parity) {
    A* xm1 = X(p - 1);
    A* x0 = X(p);
    A* xp1 = X(p + 1);
    const int width = ni;
    const int cnt = (r1 - r0) * width;
    const size_t pbase = (size_t)p * sz;
    for (int e = threadIdx.x; e < cnt; e += BLOCK) {
      int j = r0 + e / width;
      int i = e - (j - r0) * width;
      if (((i + j + p) & 1) != parity) continue;
      size_t g = pbase + (size_t)j * sy + i;
      int s = (j - jr0) * width + i;  // staged index
      A sum = A(0);
      if (p > 0) sum = sum + A(ldg(a.zp + g - sz)) * xm1[s];
      if (j > 0) sum = sum + A(ldg(a.yp + g - sy)) * x0[s - width];
      if (i > 0) sum = sum + A(ldg(a.xp + g - 1)) * x0[s - 1];
      if (i < ni - 1) sum = sum + A(ldg(a.xp + g)) * x0[s + 1];
      if (j < nj - 1) sum = sum + A(ldg(a.yp + g)) * x0[s + width];
      if (p < nk - 1) sum = sum + A(ldg(a.zp + g)) * xp1[s];
      A d = A(ldg(a.diag + g));
      x0[s] = (d != A(0)) ? gs_div(ldg(a.b + g) - sum, d) : A(0);
    }
  };

  double dot = 0.0;
  stage(k0 - 2);
  stage(k0 - 1);
  for (int p = k0 - 1; p <= kend; ++p) {
    stage(p + 1);
    __syncthreads();
    if (p >= 0 && p < nk) relax(p, jred0, jred1, 1);
    __syncthreads();
    const int q = p - 1;
    const bool out_plane = (q >= k0 && q < kend);
    if (out_plane) relax(q, j0, jout1, 0);
    __syncthreads();
    if (out_plane) {
      const A* src = X(q) + (size_t)(j0 - jr0) * ni;
      const int cnt = (jout1 - j0) * ni;
      const size_t base = (size_t)q * sz + (size_t)j0 * sy;
      for (int e = threadIdx.x; e < cnt; e += BLOCK) {
        A v = src[e];
        V o = cvt<V>(v);
        a.x_out[base + e] = o;
        if (DOT) dot += (double)ldv(&o) * (double)ldg(a.b + base + e);
      }
    }
  }
  if (DOT) {
    double s = block_sum<BLOCK>(dot, red_smem);
    if (threadIdx.x == 0) a.dot_partial[blockIdx.x + gridDim.x * blockIdx.y] = s;
  }
}

// ---------------------------------------------------------------------------
// Pipelined variant of the fused sweep for rows whose byte length is a
// multiple of 16: every array of a plane (x_in, b, diag, xp, yp, zp, and the
// coarse x for the fused prolongation) is copied into shared memory with
// cp.async one plane ahead of its use, so the relaxation phases read only
// shared memory while the next plane streams in.  Same arithmetic and the
// same schedule as rbgs_sweep_kernel (red on plane p over the one-row ring,
// black on plane p-1, store p-1), with persistent CTAs: the (row tile,
// plane) pairs of the level are split into equal contiguous ranges, one per
// CTA, so every SM streams the same number of planes.
//
// Shared-memory rings (plane q lives in slot q mod ring):
//   x 5 planes (p-2 .. p+2), b/diag/xp/yp 3 planes (p-1 .. p+1), zp 4 planes
//   (p-2 .. p+1), coarse x 5 planes.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int BLOCK>
__device__ __forceinline__ void stage_bytes(unsigned char* dst, const unsigned char* src, int bytes) {
  for (int c = threadIdx.y * blockDim.x + threadIdx.x; c < (bytes >> 4); c += BLOCK)
    cp_async16(dst + 16 * c, src + 16 * c);
}

template <typename S>
struct Sweep2Args {
  const float* x_in;
  float* x_out;
  const float* b;
  const S* diag;
  const S* xp;
  const S* yp;
  const S* zp;
  const float* xc;
  int ni, nj, nk;
  int cni, cnj;
  int tyo;         // output rows per tile; blockIdx.x = row tile
  int zlen;        // planes per CTA; blockIdx.y = plane range
  int crows_max;   // staged coarse rows per slot
  double* dot_partial;
};

// Rows staged per plane for a tile of `tyo` output rows: x needs the red ring
// and its neighbours (tyo + 4), b/diag/xp/zp the red rows (tyo + 2), yp one
// more row below them (tyo + 3).
template <typename S>
__host__ __device__ constexpr size_t sweep2_smem_bytes(int ni, int tyo, int crows, int cni) {
  return (size_t)ni * (5 * 4 * (tyo + 4) + 3 * 4 * (tyo + 2) + 3 * 2 * sizeof(S) * (tyo + 2) +
                       3 * sizeof(S) * (tyo + 3) + 4 * sizeof(S) * (tyo + 2)) +
         (size_t)5 * crows * cni * 4;
}

template <typename S, bool ZERO_X, bool PROLONG, bool DOT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) rbgs_sweep2_kernel(Sweep2Args<S> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red_smem[BLOCK / 32];
  const int ni = a.ni, nj = a.nj, nk = a.nk;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const int tyo = a.tyo;
  const int xslot = (tyo + 4) * ni, cslot = (tyo + 2) * ni, yslot = (tyo + 3) * ni;
  float* X = reinterpret_cast<float*>(smem_raw);
  float* B = X + 5 * xslot;
  S* Dg = reinterpret_cast<S*>(B + 3 * cslot);
  S* XP = Dg + 3 * cslot;
  S* ZP = XP + 3 * cslot;
  S* YP = ZP + 4 * cslot;
  float* XC = reinterpret_cast<float*>(YP + 3 * yslot);
  const int cplane = a.crows_max * a.cni;
  auto m5 = [](int q) { return (q % 5 + 5) % 5; };
  auto m3 = [](int q) { return (q % 3 + 3) % 3; };
  auto m4 = [](int q) { return q & 3; };
  const int P = (ni + 1) / 2;
  const int tx = threadIdx.x, ty = threadIdx.y, bx = blockDim.x, by = blockDim.y;
  double dot = 0.0;

  const int j0 = blockIdx.x * tyo;
  const int k0 = blockIdx.y * a.zlen;
  const int kend = min(nk, k0 + a.zlen);
  const int jout1 = min(j0 + tyo, nj);
  const int jr0 = max(j0 - 2, 0), jr1 = min(j0 + tyo + 2, nj);         // x rows
  const int jred0 = max(j0 - 1, 0), jred1 = min(j0 + tyo + 1, nj);     // b, diag, xp, zp rows
  const int jy0 = jr0;                                                  // yp rows [jy0, jred1)
  const int xrows = jr1 - jr0, crows = jred1 - jred0, yrows = jred1 - jy0;
  const int cr0 = jr0 >> 1, cr1 = ((jr1 - 1) >> 1) + 1;

  auto issue_x = [&](int q) {
    if (q < 0 || q >= nk || ZERO_X) return;
    stage_bytes<BLOCK>((unsigned char*)(X + m5(q) * xslot), (const unsigned char*)(a.x_in + q * sz + jr0 * sy),
                       xrows * ni * 4);
    if (PROLONG)
      stage_bytes<BLOCK>((unsigned char*)(XC + m5(q) * cplane),
                         (const unsigned char*)(a.xc + (size_t)(q >> 1) * a.cni * a.cnj + (size_t)cr0 * a.cni),
                         (cr1 - cr0) * a.cni * 4);
  };
  auto issue_coef = [&](int q) {
    if (q < 0 || q >= nk) return;
    const size_t o = q * sz + jred0 * sy;
    const int nb = crows * ni;
    stage_bytes<BLOCK>((unsigned char*)(B + m3(q) * cslot), (const unsigned char*)(a.b + o), nb * 4);
    stage_bytes<BLOCK>((unsigned char*)(Dg + m3(q) * cslot), (const unsigned char*)(a.diag + o),
                       nb * (int)sizeof(S));
    stage_bytes<BLOCK>((unsigned char*)(XP + m3(q) * cslot), (const unsigned char*)(a.xp + o), nb * (int)sizeof(S));
    stage_bytes<BLOCK>((unsigned char*)(YP + m3(q) * yslot), (const unsigned char*)(a.yp + q * sz + jy0 * sy),
                       yrows * ni * (int)sizeof(S));
  };
  auto issue_zp = [&](int q) {
    if (q < 0 || q >= nk) return;
    stage_bytes<BLOCK>((unsigned char*)(ZP + m4(q) * cslot), (const unsigned char*)(a.zp + q * sz + jred0 * sy),
                       crows * ni * (int)sizeof(S));
  };
  auto prolong_add = [&](int q) {
    if (!PROLONG || q < 0 || q >= nk) return;
    float* xq = X + m5(q) * xslot;
    const float* cq = XC + m5(q) * cplane;
    for (int r = ty; r < xrows; r += by) {
      const int cr = ((jr0 + r) >> 1) - cr0;
      for (int i = tx; i < ni; i += bx) xq[r * ni + i] = xq[r * ni + i] + cq[cr * a.cni + (i >> 1)];
    }
  };
  auto zero_x = [&](int q) {
    float* xq = X + m5(q) * xslot;
    for (int e = ty * bx + tx; e < xrows * ni; e += BLOCK) xq[e] = 0.0f;
  };
  // relax colour `odd` of plane p on rows [r0, r1): the reference's row sum
  // in column order (-z, -y, -x, +x, +y, +z), then (b - sum) / diag
  auto relax = [&](int p, int r0, int r1, int odd) {
    float* x0 = X + m5(p) * xslot;
    const float* xm1 = X + m5(p - 1) * xslot;
    const float* xp1 = X + m5(p + 1) * xslot;
    const float* bq = B + m3(p) * cslot;
    const S* dq = Dg + m3(p) * cslot;
    const S* xq = XP + m3(p) * cslot;
    const S* yq = YP + m3(p) * yslot;
    const S* zq = ZP + m4(p) * cslot;
    const S* zm = ZP + m4(p - 1) * cslot;
    for (int j = r0 + ty; j < r1; j += by) {
      const int sh = odd ? ((j + p + 1) & 1) : ((j + p) & 1);
      const int xrow = (j - jr0) * ni, crow = (j - jred0) * ni, yrow = (j - jy0) * ni;
      for (int m = tx; m < P; m += bx) {
        const int i = 2 * m + sh;
        if (i >= ni) continue;
        const int s = xrow + i, c = crow + i, y = yrow + i;
        float sum = 0.0f;
        if (p > 0) sum = sum + float(ldv(zm + c)) * xm1[s];
        if (j > 0) sum = sum + float(ldv(yq + y - ni)) * x0[s - ni];
        if (i > 0) sum = sum + float(ldv(xq + c - 1)) * x0[s - 1];
        if (i < ni - 1) sum = sum + float(ldv(xq + c)) * x0[s + 1];
        if (j < nj - 1) sum = sum + float(ldv(yq + y)) * x0[s + ni];
        if (p < nk - 1) sum = sum + float(ldv(zq + c)) * xp1[s];
        const float d = float(ldv(dq + c));
        x0[s] = (d != 0.0f) ? gs_div(bq[c] - sum, d) : 0.0f;
      }
    }
  };

  // prologue: x(k0-2 .. k0), coefficients (k0-1), zp(k0-2, k0-1)
  issue_x(k0 - 2);
  issue_x(k0 - 1);
  issue_x(k0);
  issue_coef(k0 - 1);
  issue_zp(k0 - 2);
  issue_zp(k0 - 1);
  cp_async_commit();
  for (int p = k0 - 1; p <= kend; ++p) {
    issue_x(p + 2);
    issue_coef(p + 1);
    issue_zp(p + 1);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    if (PROLONG || ZERO_X) {
      if (p == k0 - 1) {
        if (PROLONG) { prolong_add(k0 - 2); prolong_add(k0 - 1); }
        if (ZERO_X) { zero_x(k0 - 2); zero_x(k0 - 1); }
      }
      if (PROLONG) prolong_add(p + 1);
      if (ZERO_X) zero_x(p + 1);
      __syncthreads();
    }
    if (p >= 0 && p < nk) relax(p, jred0, jred1, 1);
    __syncthreads();
    const int q = p - 1;
    const bool out_plane = (q >= k0 && q < kend);
    if (out_plane) relax(q, j0, jout1, 0);
    __syncthreads();
    if (out_plane) {
      const float4* s4 = reinterpret_cast<const float4*>(X + m5(q) * xslot + (j0 - jr0) * ni);
      const float4* b4 = reinterpret_cast<const float4*>(B + m3(q) * cslot + (j0 - jred0) * ni);
      float4* dst = reinterpret_cast<float4*>(a.x_out + q * sz + j0 * sy);
      const int cnt4 = (jout1 - j0) * ni / 4;
      for (int e = ty * bx + tx; e < cnt4; e += BLOCK) {
        float4 v = s4[e];
        dst[e] = v;
        if (DOT) {
          float4 bb = b4[e];
          dot += (double)v.x * bb.x + (double)v.y * bb.y + (double)v.z * bb.z + (double)v.w * bb.w;
        }
      }
      if (DOT) __syncthreads();
    }
  }
  cp_async_wait0();
  if (DOT) {
    double s = block_sum<BLOCK>(dot, red_smem);
    if (threadIdx.x == 0 && threadIdx.y == 0) a.dot_partial[blockIdx.x + gridDim.x * blockIdx.y] = s;
  }
}

// ---------------------------------------------------------------------------
// Residual and restriction: b_c = R (b - A x), AlgebraicMultigrid.h:105-117.
// The residual of a row subtracts entry by entry in column order, diagonal
// included (multiply_and_subtract, sparse_matrix.h:460-480); the restriction
// adds 0.125*r over the children in ascending fine index, starting from 0
// (multiply, sparse_matrix.h:356-362).  One thread per coarse cell.
template <typename S, typename V, typename VC, bool ZERO_X>
__global__ void residual_restrict_kernel(const V* __restrict__ x, const V* __restrict__ b,
                                         const S* __restrict__ diag, const S* __restrict__ xp,
                                         const S* __restrict__ yp, const S* __restrict__ zp, VC* __restrict__ bc,
                                         int ni, int nj, int nk, int cni, int cnj, int cnk) {
  using A = typename Num<V>::Acc;
  int I = blockIdx.x * blockDim.x + threadIdx.x;
  int J = blockIdx.y * blockDim.y + threadIdx.y;
  int K = blockIdx.z;
  if (I >= cni || J >= cnj || K >= cnk) return;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  A s = A(0);
#pragma unroll
  for (int kk = 0; kk <= 1; ++kk)
#pragma unroll
    for (int jj = 0; jj <= 1; ++jj)
#pragma unroll
      for (int ii = 0; ii <= 1; ++ii) {
        int i = 2 * I + ii, j = 2 * J + jj, k = 2 * K + kk;
        if (i >= ni || j >= nj || k >= nk) continue;
        size_t g = lin3(i, j, k, ni, nj);
        A r = ldg(b + g);
        if (!ZERO_X) {
          if (k > 0) r = r - A(ldg(zp + g - sz)) * A(ldg(x + g - sz));
          if (j > 0) r = r - A(ldg(yp + g - sy)) * A(ldg(x + g - sy));
          if (i > 0) r = r - A(ldg(xp + g - 1)) * A(ldg(x + g - 1));
          r = r - A(ldg(diag + g)) * A(ldg(x + g));
          if (i < ni - 1) r = r - A(ldg(xp + g)) * A(ldg(x + g + 1));
          if (j < nj - 1) r = r - A(ldg(yp + g)) * A(ldg(x + g + sy));
          if (k < nk - 1) r = r - A(ldg(zp + g)) * A(ldg(x + g + sz));
        }
        s = s + A(0.125) * r;
      }
  bc[lin3(I, J, K, cni, cnj)] = cvt<VC>((typename Num<VC>::Acc)s);
}

// x_f += P x_c (prolongatoin, AlgebraicMultigrid.h:118-129); only used when
// a level has no post-smoothing sweep to fuse it into.
template <typename V, typename VC>
__global__ void prolong_add_kernel(V* __restrict__ xf, const VC* __restrict__ xc, int ni, int nj, int nk, int cni,
                                   int cnj) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z;
  if (i >= ni || j >= nj) return;
  size_t g = lin3(i, j, k, ni, nj);
  using A = typename Num<V>::Acc;
  xf[g] = cvt<V>(A(ldv(xf + g)) + A(ldg(xc + lin3(i >> 1, j >> 1, k >> 1, cni, cnj))));
}

// ---------------------------------------------------------------------------
// Coarsest level: `sweeps` red-black sweeps from x = 0 (AlgebraicMultigrid.h:
// 159-160, 200 sweeps), the whole level resident in shared memory of one
// CTA.  Up to 4096 unknowns (the coarsening stops at <= 16^3,
// GeometricLevelGen.h:46), six arrays of Acc.  Each thread owns the cells
// tid, tid+BLOCK, ... and decodes their coordinates, colour and neighbour
// set once, so a colour phase is a handful of shared-memory loads per cell
// and one barrier.
template <typename S, typename V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) coarsest_rbgs_kernel(const V* __restrict__ b, const S* __restrict__ diag,
                                                             const S* __restrict__ xp, const S* __restrict__ yp,
                                                             const S* __restrict__ zp, V* __restrict__ x_out,
                                                             int ni, int nj, int nk, int sweeps,
                                                             double* dot_out) {
  using A = typename Num<V>::Acc;
  constexpr int kMaxOwn = 4096 / BLOCK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = ni * nj * nk;
  A* xs = reinterpret_cast<A*>(smem_raw);
  A* bs = xs + n;
  A* ds = bs + n;
  A* xps = ds + n;
  A* yps = xps + n;
  A* zps = yps + n;
  __shared__ double red_smem[BLOCK / 32];
  for (int e = threadIdx.x; e < n; e += BLOCK) {
    xs[e] = A(0);
    bs[e] = A(ldg(b + e));
    ds[e] = A(ldg(diag + e));
    xps[e] = A(ldg(xp + e));
    yps[e] = A(ldg(yp + e));
    zps[e] = A(ldg(zp + e));
  }
  const int sy = ni, sz = ni * nj;
  // owned cells: index, colour and which of the six neighbours exist
  int own[kMaxOwn];
  int colour[kMaxOwn];
  int mask[kMaxOwn];
#pragma unroll
  for (int m = 0; m < kMaxOwn; ++m) {
    int e = threadIdx.x + m * BLOCK;
    own[m] = e;
    colour[m] = -1;
    mask[m] = 0;
    if (e < n) {
      int i = e % ni, j = (e / ni) % nj, k = e / sz;
      colour[m] = (i + j + k) & 1;
      mask[m] = (k > 0) | ((j > 0) << 1) | ((i > 0) << 2) | ((i < ni - 1) << 3) | ((j < nj - 1) << 4) |
                ((k < nk - 1) << 5);
    }
  }
  __syncthreads();
  for (int it = 0; it < sweeps; ++it) {
#pragma unroll
    for (int parity = 1; parity >= 0; --parity) {
#pragma unroll
      for (int m = 0; m < kMaxOwn; ++m) {
        if (colour[m] != parity) continue;
        const int e = own[m];
        const int f = mask[m];
        A sum = A(0);
        if (f & 1) sum = sum + zps[e - sz] * xs[e - sz];
        if (f & 2) sum = sum + yps[e - sy] * xs[e - sy];
        if (f & 4) sum = sum + xps[e - 1] * xs[e - 1];
        if (f & 8) sum = sum + xps[e] * xs[e + 1];
        if (f & 16) sum = sum + yps[e] * xs[e + sy];
        if (f & 32) sum = sum + zps[e] * xs[e + sz];
        A d = ds[e];
        xs[e] = (d != A(0)) ? gs_div(bs[e] - sum, d) : A(0);
      }
      __syncthreads();
    }
  }
  double dot = 0.0;
  for (int e = threadIdx.x; e < n; e += BLOCK) {
    V v = cvt<V>(xs[e]);
    x_out[e] = v;
    if (dot_out) dot += (double)ldv(&v) * (double)bs[e];
  }
  if (dot_out) {
    double s = block_sum<BLOCK>(dot, red_smem);
    if (threadIdx.x == 0) *dot_out = s;
  }
}

}  // namespace vflip
