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
#include "sm100.cuh"

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

// The four operator arrays of a level in one launch (convert_kernel's
// rounding): dst = [diag | xp | yp | zp], n each.
template <typename T>
__global__ void convert4_kernel(const double* __restrict__ d, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ z, T* __restrict__ dst,
                                size_t n) {
  using A = typename Num<T>::Acc;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    dst[i] = cvt<T>((A)d[i]);
    dst[n + i] = cvt<T>((A)x[i]);
    dst[2 * n + i] = cvt<T>((A)y[i]);
    dst[3 * n + i] = cvt<T>((A)z[i]);
  }
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
      if (p > 0) sum = gs_madd(sum, A(ldg(a.zp + g - sz)), xm1[s]);
      if (j > 0) sum = gs_madd(sum, A(ldg(a.yp + g - sy)), x0[s - width]);
      if (i > 0) sum = gs_madd(sum, A(ldg(a.xp + g - 1)), x0[s - 1]);
      if (i < ni - 1) sum = gs_madd(sum, A(ldg(a.xp + g)), x0[s + 1]);
      if (j < nj - 1) sum = gs_madd(sum, A(ldg(a.yp + g)), x0[s + width]);
      if (p < nk - 1) sum = gs_madd(sum, A(ldg(a.zp + g)), xp1[s]);
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
// Pipelined FP32 variant of the fused sweep for rows whose length is a
// multiple of 4 cells.  Every array of a plane region (x_in, b, diag, xp, yp,
// zp, and the coarse x of the fused prolongation) is a contiguous range of
// global memory; one thread moves each of them into shared memory with a TMA
// bulk copy (cp.async.bulk, completion on an mbarrier) one plane ahead of its
// use, so the relaxation phases read only shared memory while the next
// plane streams in.  Same arithmetic and schedule as rbgs_sweep_kernel: red
// on plane p over the tile and a one-row ring, black on plane p-1 over the
// tile, store plane p-1.
//
// Grid: (row tiles, plane ranges), sized so that every CTA is resident (one
// per SM); the CTAs of neighbouring row tiles march the same planes at the
// same time, so the halo rows one tile re-reads were just fetched by its
// neighbour and come from L2.
//
// Shared-memory rings (plane q in slot q mod ring): x 5 planes (p-2 .. p+2),
// b/diag/xp/yp 3 (p-1 .. p+1), zp 4 (p-2 .. p+1), coarse x 5.  Two mbarriers
// alternate between consecutive copy groups.  Every wait is bounded: on a
// timeout the CTA records the failure in *error, drains its own copies (again
// bounded) and returns.
template <typename S>
struct TmaSweepArgs {
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
  int tyo;        // output rows per tile; blockIdx.x = row tile
  int zlen;       // planes per CTA; blockIdx.y = plane range
  int depth;      // copy groups in flight (prefetch distance in planes), 1..3
  int crows_max;  // staged coarse rows per slot
  int l2_ahead;   // planes beyond the copy group that are prefetched into L2 (0 = none)
  double* dot_partial;
  int* error;
};

constexpr int kTmaMaxDepth = 3;

// Floats of shared memory for a tile of `tyo` output rows and prefetch depth
// D: x needs the red ring and its neighbours (tyo + 4 rows) for planes
// p-2 .. p+1 plus D in flight; b/diag/xp (tyo + 2 rows) and yp (tyo + 3)
// for planes p-1, p plus D; zp (tyo + 2) for p-2 .. p plus D; coarse x
// follows the x ring.
// Layout (4-byte units unless noted): x ring, b ring (FP32), then the
// coefficient rings diag, xp, yp, zp in elements of S (FP32 or BF16),
// then the coarse-x ring (FP32) at the next 16-byte boundary.
struct TmaLayout {
  int xslot, cslot, yslot, cplane;
  int oX, oB, oC;        // float offsets: x ring, b ring, start of the coefficient region
  int cD, cXP, cYP, cZP; // S-element offsets inside the coefficient region
  int oXC;               // float offset of the coarse-x ring
  size_t bytes;
};

template <typename S>
__host__ __device__ inline TmaLayout tma_layout(int ni, int tyo, int depth, int crows, int cni) {
  TmaLayout L;
  const int RX = 4 + depth, RC = 2 + depth, RZ = 3 + depth;
  L.xslot = (tyo + 4) * ni;
  L.cslot = (tyo + 2) * ni;
  L.yslot = (tyo + 3) * ni;
  L.cplane = crows * cni;
  L.oX = 0;
  L.oB = L.oX + RX * L.xslot;
  L.oC = L.oB + RC * L.cslot;
  L.cD = 0;
  L.cXP = L.cD + RC * L.cslot;
  L.cYP = L.cXP + RC * L.cslot;
  L.cZP = L.cYP + RC * L.yslot;
  const size_t coef_bytes = (size_t)(L.cZP + RZ * L.cslot) * sizeof(S);
  const size_t xc_byte = ((size_t)L.oC * 4 + coef_bytes + 15) / 16 * 16;
  L.oXC = (int)(xc_byte / 4);
  L.bytes = xc_byte + (size_t)RX * L.cplane * 4;
  return L;
}


// Four consecutive elements of a shared-memory row as floats (16-byte
// aligned FP32 or 8-byte aligned BF16).
__device__ __forceinline__ float4 ld4f(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ld4f(const __nv_bfloat16* p) {
  const uint2 u = *reinterpret_cast<const uint2*>(p);
  const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&u.x), b = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
  const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
  return make_float4(fa.x, fa.y, fb.x, fb.y);
}
// (the FP64 instantiation of the pipelined kernel is compiled but never launched)
__device__ __forceinline__ float4 ld4f(const double* p) {
  return make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
}
template <int K>
__device__ __forceinline__ float c4(const float4& v) {
  return K == 0 ? v.x : K == 1 ? v.y : K == 2 ? v.z : v.w;
}
// Relaxation of cell K of a quad of four consecutive cells (i0 .. i0+3):
// the reference's row sum in column order (-z, -y, -x, +x, +y, +z), then
// (b - sum) / diag.  xl/xr are x at i0-1 / i0+4, cxl is +x coupling of i0-1.
template <int K>
__device__ __forceinline__ float relax_quad_cell(bool zlo, bool zhi, bool ylo, bool yhi, bool xlo, bool xhi,
                                                 const float4& xc, const float4& xym, const float4& xyp,
                                                 const float4& xzm, const float4& xzp, float xl, float xr,
                                                 const float4& bb, const float4& dd, const float4& cx, float cxl,
                                                 const float4& cyp, const float4& cym, const float4& czp,
                                                 const float4& czm) {
  constexpr int KL = K > 0 ? K - 1 : 0, KR = K < 3 ? K + 1 : 3;
  float sum = 0.0f;
  if (zlo) sum = gs_madd(sum, c4<K>(czm), c4<K>(xzm));
  if (ylo) sum = gs_madd(sum, c4<K>(cym), c4<K>(xym));
  if (xlo) sum = gs_madd(sum, (K == 0 ? cxl : c4<KL>(cx)), (K == 0 ? xl : c4<KL>(xc)));
  if (xhi) sum = gs_madd(sum, c4<K>(cx), (K == 3 ? xr : c4<KR>(xc)));
  if (yhi) sum = gs_madd(sum, c4<K>(cyp), c4<K>(xyp));
  if (zhi) sum = gs_madd(sum, c4<K>(czp), c4<K>(xzp));
  const float d = c4<K>(dd);
  return (d != 0.0f) ? gs_div(c4<K>(bb) - sum, d) : 0.0f;
}

template <typename S, bool ZERO_X, bool PROLONG, bool DOT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) rbgs_sweep_tma_kernel(TmaSweepArgs<S> a) {
  extern __shared__ __align__(128) float sm[];
  constexpr int NB = kTmaMaxDepth + 2;  // mbarrier ring
  __shared__ __align__(8) unsigned long long bars[NB];
  __shared__ double red_smem[BLOCK / 32];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int ni = a.ni, nj = a.nj, nk = a.nk, tyo = a.tyo, D = a.depth;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const TmaLayout Ly = tma_layout<S>(ni, tyo, D, a.crows_max, a.cni);
  const int xslot = Ly.xslot, cslot = Ly.cslot, yslot = Ly.yslot, cplane = Ly.cplane;
  const int RX = 4 + D, RC = 2 + D, RZ = 3 + D;  // ring lengths
  const int oX = Ly.oX, oB = Ly.oB, oXC = Ly.oXC;
  const int oD = Ly.cD, oXP = Ly.cXP, oYP = Ly.cYP, oZP = Ly.cZP;  // in elements of S
  const S* cs = reinterpret_cast<const S*>(sm + Ly.oC);
  const unsigned cbase_b = 4u * (unsigned)Ly.oC;  // byte offset of the coefficient region
  constexpr unsigned ES = sizeof(S);
  const int tx = threadIdx.x, ty = threadIdx.y, bx = blockDim.x, by = blockDim.y;

  const int j0 = blockIdx.x * tyo;
  const int k0 = blockIdx.y * a.zlen;
  const int kend = min(nk, k0 + a.zlen);
  const int jout1 = min(j0 + tyo, nj);
  const int jr0 = max(j0 - 2, 0), jr1 = min(j0 + tyo + 2, nj);      // x rows
  const int jred0 = max(j0 - 1, 0), jred1 = min(j0 + tyo + 1, nj);  // b, diag, xp, zp rows
  const int jy0 = jr0;                                               // yp rows [jy0, jred1)
  const int xrows = jr1 - jr0, crows = jred1 - jred0, yrows = jred1 - jy0;
  const int cr0 = jr0 >> 1, cr1 = ((jr1 - 1) >> 1) + 1;

  const unsigned sbase = smem_u32(sm);
  const unsigned bar_base = smem_u32(&bars[0]);
  if (tid == 0) {
    for (int q = 0; q < NB; ++q) mbar_init(bar_base + 8u * q, 1);
    mbar_init_fence();
  }
  __syncthreads();

  // Ring slots.  Plane q lives in slot q mod ring; the loop carries the slot
  // of the current plane p in each ring and steps it by one per plane, so no
  // division runs inside the loop.
  auto wrap = [](int v, int r) { return v >= r ? v - r : (v < 0 ? v + r : v); };
  const int p0 = k0 - 1;
  int px = ((p0 % RX) + RX) % RX, pc = ((p0 % RC) + RC) % RC, pz = ((p0 % RZ) + RZ) % RZ;

  // thread 0: copy group g on mbarrier g % NB, phase (g / NB) & 1: x planes
  // qx0/qx1 into x slots sx0/sx1, coefficient plane qc into slot sc, zp plane
  // qz into slot szs (planes out of the domain are skipped)
  auto issue = [&](int g, int qx0, int sx0, int qx1, int sx1, int qc, int sc, int qz, int szs) {
    const unsigned bar = bar_base + 8u * (unsigned)(g % NB);
    const bool hx0 = !ZERO_X && qx0 >= 0 && qx0 < nk, hx1 = !ZERO_X && qx1 >= 0 && qx1 < nk;
    const bool hc = qc >= 0 && qc < nk, hz = qz >= 0 && qz < nk;
    const unsigned xb = xrows * ni * 4 + (PROLONG ? (cr1 - cr0) * a.cni * 4 : 0);
    const unsigned bytes = (hx0 ? xb : 0) + (hx1 ? xb : 0) +
                           (hc ? crows * ni * 4 + (2 * crows + yrows) * ni * ES : 0) + (hz ? crows * ni * ES : 0);
    fence_proxy_async();
    mbar_expect_tx(bar, bytes);
    for (int h = 0; h < 2; ++h) {
      const int qx = h ? qx1 : qx0, sx = h ? sx1 : sx0;
      if (!(h ? hx1 : hx0)) continue;
      tma_bulk_g2s(sbase + 4u * (oX + sx * xslot), a.x_in + qx * sz + jr0 * sy, xrows * ni * 4, bar);
      if (PROLONG)
        tma_bulk_g2s(sbase + 4u * (oXC + sx * cplane), a.xc + (size_t)(qx >> 1) * a.cni * a.cnj + (size_t)cr0 * a.cni,
                     (cr1 - cr0) * a.cni * 4, bar);
    }
    if (hc) {
      const size_t o = qc * sz + jred0 * sy;
      tma_bulk_g2s(sbase + 4u * (oB + sc * cslot), a.b + o, crows * ni * 4, bar);
      tma_bulk_g2s(sbase + cbase_b + ES * (oD + sc * cslot), a.diag + o, crows * ni * ES, bar);
      tma_bulk_g2s(sbase + cbase_b + ES * (oXP + sc * cslot), a.xp + o, crows * ni * ES, bar);
      tma_bulk_g2s(sbase + cbase_b + ES * (oYP + sc * yslot), a.yp + qc * sz + jy0 * sy, yrows * ni * ES, bar);
    }
    if (hz)
      tma_bulk_g2s(sbase + cbase_b + ES * (oZP + szs * cslot), a.zp + qz * sz + jred0 * sy, crows * ni * ES, bar);
    // The same plane region l2_ahead planes further on, into L2 only: the
    // shared-memory ring holds one copy group in flight, which leaves HBM
    // idle for a copy's latency every plane; the prefetches keep it busy and
    // turn the later bulk copies into L2 hits.
    const int qp = (hc ? qc : qx0) + a.l2_ahead;
    if (a.l2_ahead > 0 && qp < nk && qp >= 0) {
      if (!ZERO_X) tma_prefetch_l2(a.x_in + (qp + 1 < nk ? qp + 1 : qp) * sz + jr0 * sy, xrows * ni * 4);
      const size_t o = qp * sz + jred0 * sy;
      tma_prefetch_l2(a.b + o, crows * ni * 4);
      tma_prefetch_l2(a.diag + o, crows * ni * ES);
      tma_prefetch_l2(a.xp + o, crows * ni * ES);
      tma_prefetch_l2(a.yp + qp * sz + jy0 * sy, yrows * ni * ES);
      tma_prefetch_l2(a.zp + o, crows * ni * ES);
    }
  };
  // all threads: wait for group g; block-uniform result
  auto wait_group = [&](int g) -> bool {
    const bool ok = mbar_wait_bounded(bar_base + 8u * (unsigned)(g % NB), (unsigned)((g / NB) & 1));
    return __syncthreads_and(ok) != 0;
  };

  // relax colour `odd` of plane p on rows [r0, r1) (slot offsets given).
  // A thread takes quads of four consecutive cells (rows are multiples of 4
  // long) and updates the quad's two cells of that colour from 16-byte
  // loads; each cell's arithmetic is the reference's, in its order.
  // With `store` (the black pass of an output plane) each thread also writes
  // its whole quad to x_out - two new black values and the two red values
  // finished one step earlier - and adds the quad to the fused z.r.
  double dot = 0.0;
  auto relax = [&](int p, int r0, int r1, int odd, int x0, int xm1, int xp1, int cb, int cd, int cx, int cy, int cz,
                   int czm, bool store) {
    const bool zlo = p > 0, zhi = p < nk - 1;
    const int Q = ni >> 2;
    float* outp = a.x_out + (size_t)p * sz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = r0 + ty; j < r1; j += by) {
      const int sh = (j + p + odd) & 1;
      const int xr = (j - jr0) * ni, cr = (j - jred0) * ni, yr = (j - jy0) * ni;
      const bool ylo = j > 0, yhi = j < nj - 1;
      for (int q = tx; q < Q; q += bx) {
        const int i0 = 4 * q;
        const int s = xr + i0, c = cr + i0, y = yr + i0;
        const float4 xc = ld4f(sm + x0 + s);
        const float4 xym = ylo ? ld4f(sm + x0 + s - ni) : z4, xyp = yhi ? ld4f(sm + x0 + s + ni) : z4;
        const float4 xzm = zlo ? ld4f(sm + xm1 + s) : z4, xzp = zhi ? ld4f(sm + xp1 + s) : z4;
        const float4 bb = ld4f(sm + cb + c), dd = ld4f(cs + cd + c), cxv = ld4f(cs + cx + c);
        const float4 cyp = ld4f(cs + cy + y), cym = ylo ? ld4f(cs + cy + y - ni) : z4;
        const float4 czp = ld4f(cs + cz + c), czmv = zlo ? ld4f(cs + czm + c) : z4;
        if (sh == 0) {
          const float xl = i0 > 0 ? sm[x0 + s - 1] : 0.0f;
          const float cxl = i0 > 0 ? float(ldv(cs + cx + c - 1)) : 0.0f;
          const float v0 = relax_quad_cell<0>(zlo, zhi, ylo, yhi, i0 > 0, i0 < ni - 1, xc, xym, xyp, xzm, xzp, xl,
                                              0.0f, bb, dd, cxv, cxl, cyp, cym, czp, czmv);
          const float v2 = relax_quad_cell<2>(zlo, zhi, ylo, yhi, true, i0 + 2 < ni - 1, xc, xym, xyp, xzm, xzp,
                                              0.0f, 0.0f, bb, dd, cxv, 0.0f, cyp, cym, czp, czmv);
          sm[x0 + s] = v0;
          sm[x0 + s + 2] = v2;
          if (store) {
            const float4 o = make_float4(v0, xc.y, v2, xc.w);
            *reinterpret_cast<float4*>(outp + (size_t)j * sy + i0) = o;
            if (DOT) dot += (double)o.x * bb.x + (double)o.y * bb.y + (double)o.z * bb.z + (double)o.w * bb.w;
          }
        } else {
          const float xr4 = i0 + 4 < ni ? sm[x0 + s + 4] : 0.0f;
          const float v1 = relax_quad_cell<1>(zlo, zhi, ylo, yhi, true, i0 + 1 < ni - 1, xc, xym, xyp, xzm, xzp,
                                              0.0f, 0.0f, bb, dd, cxv, 0.0f, cyp, cym, czp, czmv);
          const float v3 = relax_quad_cell<3>(zlo, zhi, ylo, yhi, true, i0 + 3 < ni - 1, xc, xym, xyp, xzm, xzp,
                                              0.0f, xr4, bb, dd, cxv, 0.0f, cyp, cym, czp, czmv);
          sm[x0 + s + 1] = v1;
          sm[x0 + s + 3] = v3;
          if (store) {
            const float4 o = make_float4(xc.x, v1, xc.z, v3);
            *reinterpret_cast<float4*>(outp + (size_t)j * sy + i0) = o;
            if (DOT) dot += (double)o.x * bb.x + (double)o.y * bb.y + (double)o.z * bb.z + (double)o.w * bb.w;
          }
        }
      }
    }
  };
  auto prolong_add = [&](int q, int slot) {
    if (q < 0 || q >= nk) return;
    const int xq = oX + slot * xslot, cq = oXC + slot * cplane;
    for (int r = ty; r < xrows; r += by) {
      const int crr = ((jr0 + r) >> 1) - cr0;
      for (int i = tx; i < ni; i += bx) sm[xq + r * ni + i] = sm[xq + r * ni + i] + sm[cq + crr * a.cni + (i >> 1)];
    }
  };
  auto zero_x = [&](int slot) {
    const int xq = oX + slot * xslot;
    for (int e = tid; e < xrows * ni; e += BLOCK) sm[xq + e] = 0.0f;
  };

  // Copy groups: G0 = x(k0-2), x(k0-1), zp(k0-2); then H(q) for q >= k0-1
  // carries x(q+1), coefficients (q), zp(q) and is group q - k0 + 2.  The
  // step for plane p waits for H(p) (and G0 first), then issues H(p+D), so
  // D groups stream in during its relaxation.
  bool failed = false;
  int issued = 1;
  if (tid == 0) issue(0, p0 - 1, wrap(px - 1, RX), p0, px, -1, 0, p0 - 1, wrap(pz - 1, RZ));
  for (int d = 0; d < D && p0 + d <= kend; ++d) {
    if (tid == 0) issue(1 + d, p0 + d + 1, wrap(px + d + 1, RX), -1, 0, p0 + d, wrap(pc + d, RC), p0 + d,
                        wrap(pz + d, RZ));
    issued = 2 + d;
  }
  for (int p = p0; p <= kend; ++p) {
    if (p == p0 && !wait_group(0)) { failed = true; break; }
    if (!wait_group(p - k0 + 2)) { failed = true; break; }
    if (p + D <= kend) {
      if (tid == 0) issue(p + D - k0 + 2, p + D + 1, wrap(px + D + 1, RX), -1, 0, p + D, wrap(pc + D, RC), p + D,
                          wrap(pz + D, RZ));
      issued = p + D - k0 + 3;
    }
    const int sxm2 = wrap(px - 2, RX), sxm1 = wrap(px - 1, RX), sxp1 = wrap(px + 1, RX);
    const int scm1 = wrap(pc - 1, RC);
    const int szm2 = wrap(pz - 2, RZ), szm1 = wrap(pz - 1, RZ);
    if (PROLONG || ZERO_X) {
      if (p == p0) {
        if (PROLONG) { prolong_add(p - 1, sxm1); prolong_add(p, px); }
        if (ZERO_X) { zero_x(sxm1); zero_x(px); }
      }
      if (PROLONG) prolong_add(p + 1, sxp1);
      if (ZERO_X) zero_x(sxp1);
      __syncthreads();
    }
    if (p >= 0 && p < nk)
      relax(p, jred0, jred1, 1, oX + px * xslot, oX + sxm1 * xslot, oX + sxp1 * xslot, oB + pc * cslot,
            oD + pc * cslot, oXP + pc * cslot, oYP + pc * yslot, oZP + pz * cslot, oZP + szm1 * cslot, false);
    __syncthreads();
    // black pass of plane p-1 with the quads stored as they finish; the next
    // step's wait barrier orders it before any slot it reads is refilled
    const int q = p - 1;
    if (q >= k0 && q < kend)
      relax(q, j0, jout1, 0, oX + sxm1 * xslot, oX + sxm2 * xslot, oX + px * xslot, oB + scm1 * cslot,
            oD + scm1 * cslot, oXP + scm1 * cslot, oYP + scm1 * yslot, oZP + szm1 * cslot, oZP + szm2 * cslot, true);
    px = wrap(px + 1, RX);
    pc = wrap(pc + 1, RC);
    pz = wrap(pz + 1, RZ);
  }
  if (failed) {
    if (tid == 0) atomicExch(a.error, 1);
    // drain: every issued group must land before the CTA's shared memory is
    // released (bounded again)
    for (int g = max(0, issued - NB); g < issued; ++g)
      mbar_wait_bounded(bar_base + 8u * (unsigned)(g % NB), (unsigned)((g / NB) & 1));
    return;
  }
  if (DOT) {
    double s = block_sum<BLOCK>(dot, red_smem);
    if (tid == 0) a.dot_partial[blockIdx.x + gridDim.x * blockIdx.y] = s;
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
          // every operand loaded before the row's subtractions (neighbours
          // outside the level at a clamped, in-range address, then unused),
          // so a child's loads are in flight together; the subtractions keep
          // their order and roundings
          const bool zl = k > 0, yl = j > 0, xl = i > 0, xh = i < ni - 1, yh = j < nj - 1, zh = k < nk - 1;
          const A czm = A(ldg(zp + (zl ? g - sz : g))), xzm = A(ldg(x + (zl ? g - sz : g)));
          const A cym = A(ldg(yp + (yl ? g - sy : g))), xym = A(ldg(x + (yl ? g - sy : g)));
          const A cxm = A(ldg(xp + (xl ? g - 1 : g))), xxm = A(ldg(x + (xl ? g - 1 : g)));
          const A cd = A(ldg(diag + g)), xc = A(ldg(x + g));
          const A cxp = A(ldg(xp + g)), xxp = A(ldg(x + (xh ? g + 1 : g)));
          const A cyp = A(ldg(yp + g)), xyp = A(ldg(x + (yh ? g + sy : g)));
          const A czp = A(ldg(zp + g)), xzp = A(ldg(x + (zh ? g + sz : g)));
          if (zl) r = r - czm * xzm;
          if (yl) r = r - cym * xym;
          if (xl) r = r - cxm * xxm;
          r = r - cd * xc;
          if (xh) r = r - cxp * xxp;
          if (yh) r = r - cyp * xyp;
          if (zh) r = r - czp * xzp;
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
                                                             double* dot_out, const int* skip_if_set) {
  // the FP64 direct solve of this level ran instead (coarse_direct.cuh)
  if (skip_if_set && *skip_if_set) return;
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
  // owned cells tid + m*BLOCK: bits 0-5 say which of the six neighbours
  // exist, bits 6-7 hold the colour (0 or 1) or 2 for "no cell"
  int mask[kMaxOwn];
#pragma unroll
  for (int m = 0; m < kMaxOwn; ++m) {
    int e = threadIdx.x + m * BLOCK;
    mask[m] = 2 << 6;
    if (e < n) {
      int i = e % ni, j = (e / ni) % nj, k = e / sz;
      mask[m] = (k > 0) | ((j > 0) << 1) | ((i > 0) << 2) | ((i < ni - 1) << 3) | ((j < nj - 1) << 4) |
                ((k < nk - 1) << 5) | (((i + j + k) & 1) << 6);
    }
  }
  __syncthreads();
  if (sizeof(A) == 4) {
    // FP32: each owned cell's couplings, diagonal and rhs stay in registers
    // (a missing neighbour gets coupling 0 and reads the cell itself), so a
    // colour phase is six shared loads per cell and one barrier
    A c[kMaxOwn][6], dd[kMaxOwn], bb[kMaxOwn];
#pragma unroll
    for (int m = 0; m < kMaxOwn; ++m) {
      const int e = (threadIdx.x + m * BLOCK) < n ? (threadIdx.x + m * BLOCK) : 0;
      const int f = mask[m];
      c[m][0] = (f & 1) ? zps[e - sz] : A(0);
      c[m][1] = (f & 2) ? yps[e - sy] : A(0);
      c[m][2] = (f & 4) ? xps[e - 1] : A(0);
      c[m][3] = (f & 8) ? xps[e] : A(0);
      c[m][4] = (f & 16) ? yps[e] : A(0);
      c[m][5] = (f & 32) ? zps[e] : A(0);
      dd[m] = ds[e];
      bb[m] = bs[e];
    }
    for (int it = 0; it < sweeps; ++it) {
#pragma unroll
      for (int parity = 1; parity >= 0; --parity) {
#pragma unroll
        for (int m = 0; m < kMaxOwn; ++m) {
          if ((mask[m] >> 6) != parity) continue;
          const int e = threadIdx.x + m * BLOCK;
          const int f = mask[m];
          A sum = A(0);
          sum = gs_madd(sum, c[m][0], xs[(f & 1) ? e - sz : e]);
          sum = gs_madd(sum, c[m][1], xs[(f & 2) ? e - sy : e]);
          sum = gs_madd(sum, c[m][2], xs[(f & 4) ? e - 1 : e]);
          sum = gs_madd(sum, c[m][3], xs[(f & 8) ? e + 1 : e]);
          sum = gs_madd(sum, c[m][4], xs[(f & 16) ? e + sy : e]);
          sum = gs_madd(sum, c[m][5], xs[(f & 32) ? e + sz : e]);
          xs[e] = (dd[m] != A(0)) ? gs_div(bb[m] - sum, dd[m]) : A(0);
        }
        __syncthreads();
      }
    }
  } else {
    for (int it = 0; it < sweeps; ++it) {
#pragma unroll
      for (int parity = 1; parity >= 0; --parity) {
#pragma unroll
        for (int m = 0; m < kMaxOwn; ++m) {
          if ((mask[m] >> 6) != parity) continue;
          const int e = threadIdx.x + m * BLOCK;
          const int f = mask[m];
          A sum = A(0);
          if (f & 1) sum = gs_madd(sum, zps[e - sz], xs[e - sz]);
          if (f & 2) sum = gs_madd(sum, yps[e - sy], xs[e - sy]);
          if (f & 4) sum = gs_madd(sum, xps[e - 1], xs[e - 1]);
          if (f & 8) sum = gs_madd(sum, xps[e], xs[e + 1]);
          if (f & 16) sum = gs_madd(sum, yps[e], xs[e + sy]);
          if (f & 32) sum = gs_madd(sum, zps[e], xs[e + sz]);
          A d = ds[e];
          xs[e] = (d != A(0)) ? gs_div(bs[e] - sum, d) : A(0);
        }
        __syncthreads();
      }
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
