// Grid sampling, semi-Lagrangian advection and the FLIP particle<->grid
// transfers.
//
// Sampling follows Buffer3D::sample_linear/at (Smoke_Solver/fluid_buffer3D.h:
// 205-248): world -> grid coordinates in double, floor, clamp-to-edge, three
// levels of lerp in double, rounded to float at the end.  Keeping that FP64
// arithmetic makes advection and G2P bit-identical to the reference.
//
// P2G is a sort-by-cell gather: particles are bucketed by cell with a
// counting sort whose buckets are then put into ascending particle order, so
// each face node sums its neighbours' contributions in exactly the order
// SmokeSolver3D::particle_to_grid does (27 buckets in (k,j,i) order, bucket
// contents in insertion order, Smoke_solver3D.cpp:1477-1502).  The sums are
// deterministic and bit-identical to the reference.
#pragma once
#include <climits>
#include "common.cuh"

namespace vflip {

struct GridView {
  const float* d;
  int nx, ny, nz;
  double h, ox, oy, oz;
  double inv_h;  // 1/h when h is a power of two (then x*inv_h == x/h exactly), else 0
};

// x / h exactly as IEEE division; a multiplication when h is a power of two
__device__ __forceinline__ double div_h(double x, const GridView& g) { return g.inv_h != 0.0 ? x * g.inv_h : x / g.h; }

__device__ __forceinline__ int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

__device__ __forceinline__ double lerp_d(double a, double b, double c) { return (1.0 - c) * a + c * b; }

// The eight corners share three clamped coordinate pairs; addresses are
// 32-bit element offsets (every grid here has fewer than 2^31 elements).
__device__ __forceinline__ float sample_linear(const GridView& g, double wx, double wy, double wz) {
  double gx = div_h(wx, g) + g.ox, gy = div_h(wy, g) + g.oy, gz = div_h(wz, g) + g.oz;
  int i = (int)floor(gx), j = (int)floor(gy), k = (int)floor(gz);
  double cx = gx - (double)i, cy = gy - (double)j, cz = gz - (double)k;
  const int i0 = clampi(i, g.nx - 1), i1 = clampi(i + 1, g.nx - 1);
  const int sy = g.nx, sz = g.nx * g.ny;
  const int j0 = clampi(j, g.ny - 1) * sy, j1 = clampi(j + 1, g.ny - 1) * sy;
  const int k0 = clampi(k, g.nz - 1) * sz, k1 = clampi(k + 1, g.nz - 1) * sz;
  const float* d = g.d;
  const double a000 = __ldg(d + (i0 + j0 + k0)), a100 = __ldg(d + (i1 + j0 + k0));
  const double a010 = __ldg(d + (i0 + j1 + k0)), a110 = __ldg(d + (i1 + j1 + k0));
  const double a001 = __ldg(d + (i0 + j0 + k1)), a101 = __ldg(d + (i1 + j0 + k1));
  const double a011 = __ldg(d + (i0 + j1 + k1)), a111 = __ldg(d + (i1 + j1 + k1));
  double v1 = lerp_d(lerp_d(a000, a100, cx), lerp_d(a010, a110, cx), cy);
  double v2 = lerp_d(lerp_d(a001, a101, cx), lerp_d(a011, a111, cx), cy);
  return (float)lerp_d(v1, v2, cz);
}

// FP32 variant of sample_linear for the FP32/mixed precision modes: the
// same corners and lerp structure with the world->grid transform and the
// lerps in float (within a few ulp of the FP64 form, not bit-identical).
__device__ __forceinline__ float lerp_f(float a, float b, float c) { return __fmaf_rn(c, b - a, a); }

__device__ __forceinline__ float sample_linear_f(const GridView& g, float wx, float wy, float wz) {
  const float ih = (float)(g.inv_h != 0.0 ? g.inv_h : 1.0 / g.h);
  float gx = __fmaf_rn(wx, ih, (float)g.ox), gy = __fmaf_rn(wy, ih, (float)g.oy), gz = __fmaf_rn(wz, ih, (float)g.oz);
  float fi = floorf(gx), fj = floorf(gy), fk = floorf(gz);
  int i = (int)fi, j = (int)fj, k = (int)fk;
  float cx = gx - fi, cy = gy - fj, cz = gz - fk;
  const int i0 = clampi(i, g.nx - 1), i1 = clampi(i + 1, g.nx - 1);
  const int sy = g.nx, sz = g.nx * g.ny;
  const int j0 = clampi(j, g.ny - 1) * sy, j1 = clampi(j + 1, g.ny - 1) * sy;
  const int k0 = clampi(k, g.nz - 1) * sz, k1 = clampi(k + 1, g.nz - 1) * sz;
  const float* d = g.d;
  float v1 = lerp_f(lerp_f(__ldg(d + (i0 + j0 + k0)), __ldg(d + (i1 + j0 + k0)), cx),
                    lerp_f(__ldg(d + (i0 + j1 + k0)), __ldg(d + (i1 + j1 + k0)), cx), cy);
  float v2 = lerp_f(lerp_f(__ldg(d + (i0 + j0 + k1)), __ldg(d + (i1 + j0 + k1)), cx),
                    lerp_f(__ldg(d + (i0 + j1 + k1)), __ldg(d + (i1 + j1 + k1)), cx), cy);
  return lerp_f(v1, v2, cz);
}

// SubDomainSolver::advect_field, sub_domain.cpp:191-235: RK2 midpoint
// backtrace through the MAC velocity, then a trilinear sample of the field.
// The field's node (i,j,k) sits at world ((i-ox)h, (j-oy)h, (k-oz)h).  A
// second field on the same grid (f2.d != nullptr) shares the backtrace.
// Each thread carries two nodes through the three dependent gather rounds
// so that their loads overlap.
struct Backtrace {
  float px, py, pz;
};

__device__ __forceinline__ void node_world(const GridView& f, size_t e, float h, float& wx, float& wy, float& wz) {
  int i, j, k;
  decode3(e, f.nx, f.ny, i, j, k);
  wx = (float)(((double)(float)i - f.ox) * (double)h);
  wy = (float)(((double)(float)j - f.oy) * (double)h);
  wz = (float)(((double)(float)k - f.oz) * (double)h);
}

// Each block owns a contiguous run of `per_block` nodes (so the blocks in
// flight cover a compact slab and the gathers of neighbouring blocks hit
// L2), walked two nodes per thread at a time.
template <bool EXACT>
__device__ __forceinline__ float smp(const GridView& g, float x, float y, float z) {
  return EXACT ? sample_linear(g, x, y, z) : sample_linear_f(g, x, y, z);
}

// EXACT: the reference's arithmetic (FP64 transform and lerps, FP64 midpoint
// step), bit-identical to SubDomainSolver::advect_field; otherwise the same
// scheme in FP32 (FP32 contexts launch advect_rk2_f_kernel, its values bit
// for bit with less work per sample).
template <bool EXACT>
__global__ void advect_rk2_kernel(GridView u, GridView v, GridView w, GridView f, float* __restrict__ out,
                                  GridView f2, float* __restrict__ out2, float h, float dt, int per_block) {
  const size_t n = (size_t)f.nx * f.ny * f.nz;
  const size_t stride = blockDim.x;
  const double hdt = 0.5 * (double)dt;
  const size_t beg = (size_t)blockIdx.x * per_block;
  const size_t end = beg + per_block < n ? beg + per_block : n;
  for (size_t e0 = beg + threadIdx.x; e0 < end; e0 += 2 * stride) {
    const size_t e1 = e0 + stride;
    const bool two = e1 < end;
    float wx0, wy0, wz0, wx1 = 0, wy1 = 0, wz1 = 0;
    node_world(f, e0, h, wx0, wy0, wz0);
    if (two) node_world(f, e1, h, wx1, wy1, wz1);
    float a0 = smp<EXACT>(u, wx0, wy0, wz0), b0 = smp<EXACT>(v, wx0, wy0, wz0), c0 = smp<EXACT>(w, wx0, wy0, wz0);
    float a1 = 0, b1 = 0, c1 = 0;
    if (two) {
      a1 = smp<EXACT>(u, wx1, wy1, wz1);
      b1 = smp<EXACT>(v, wx1, wy1, wz1);
      c1 = smp<EXACT>(w, wx1, wy1, wz1);
    }
    float px0, py0, pz0, px1, py1, pz1;
    if (EXACT) {
      px0 = (float)((double)wx0 - hdt * (double)a0);
      py0 = (float)((double)wy0 - hdt * (double)b0);
      pz0 = (float)((double)wz0 - hdt * (double)c0);
      px1 = (float)((double)wx1 - hdt * (double)a1);
      py1 = (float)((double)wy1 - hdt * (double)b1);
      pz1 = (float)((double)wz1 - hdt * (double)c1);
    } else {
      const float hf = 0.5f * dt;
      px0 = wx0 - hf * a0; py0 = wy0 - hf * b0; pz0 = wz0 - hf * c0;
      px1 = wx1 - hf * a1; py1 = wy1 - hf * b1; pz1 = wz1 - hf * c1;
    }
    a0 = smp<EXACT>(u, px0, py0, pz0);
    b0 = smp<EXACT>(v, px0, py0, pz0);
    c0 = smp<EXACT>(w, px0, py0, pz0);
    if (two) {
      a1 = smp<EXACT>(u, px1, py1, pz1);
      b1 = smp<EXACT>(v, px1, py1, pz1);
      c1 = smp<EXACT>(w, px1, py1, pz1);
    }
    px0 = wx0 - dt * a0;
    py0 = wy0 - dt * b0;
    pz0 = wz0 - dt * c0;
    px1 = wx1 - dt * a1;
    py1 = wy1 - dt * b1;
    pz1 = wz1 - dt * c1;
    out[e0] = smp<EXACT>(f, px0, py0, pz0);
    if (out2) out2[e0] = smp<EXACT>(f2, px0, py0, pz0);
    if (two) {
      out[e1] = smp<EXACT>(f, px1, py1, pz1);
      if (out2) out2[e1] = smp<EXACT>(f2, px1, py1, pz1);
    }
  }
}

// ---- the FP32 form (advect_rk2_kernel<false>'s values bit for bit) with
// the per-sample work cut down: each grid's float transform (1/h, offsets)
// is computed once on the host, and the staggered u, v, w grids share the
// axis coordinates they have in common (x of v and w, y of u and w, z of u
// and v: same offset and extent), so a velocity sample at one point takes
// six floor/clamp axis evaluations instead of nine.
struct GridF {
  const float* d;
  int nx, ny, nz;
  float ox, oy, oz;  // (float) of the grid's offsets
};

struct AxisF {
  int i0, i1;  // clamped corner indices
  float c;     // fraction
};

__device__ __forceinline__ AxisF axis_f(float w, float ih, float o, int n) {
  const float g = __fmaf_rn(w, ih, o);
  const float f = floorf(g);
  const int i = (int)f;
  return AxisF{clampi(i, n - 1), clampi(i + 1, n - 1), g - f};
}

// sample_linear_f's corners and lerps from precomputed axes (sy, sz: strides)
__device__ __forceinline__ float tri_f(const float* __restrict__ d, int sy, int sz, const AxisF& x, const AxisF& y,
                                       const AxisF& z) {
  const int i0 = x.i0, i1 = x.i1, j0 = y.i0 * sy, j1 = y.i1 * sy, k0 = z.i0 * sz, k1 = z.i1 * sz;
  float v1 = lerp_f(lerp_f(__ldg(d + (i0 + j0 + k0)), __ldg(d + (i1 + j0 + k0)), x.c),
                    lerp_f(__ldg(d + (i0 + j1 + k0)), __ldg(d + (i1 + j1 + k0)), x.c), y.c);
  float v2 = lerp_f(lerp_f(__ldg(d + (i0 + j0 + k1)), __ldg(d + (i1 + j0 + k1)), x.c),
                    lerp_f(__ldg(d + (i0 + j1 + k1)), __ldg(d + (i1 + j1 + k1)), x.c), y.c);
  return lerp_f(v1, v2, z.c);
}

__device__ __forceinline__ float grid_f(const GridF& g, float ih, float wx, float wy, float wz) {
  return tri_f(g.d, g.nx, g.nx * g.ny, axis_f(wx, ih, g.ox, g.nx), axis_f(wy, ih, g.oy, g.ny),
               axis_f(wz, ih, g.oz, g.nz));
}

// u, v, w of the MAC grid of ni x nj x nk cells at one point (u: offsets
// (0.5, 0, 0), extent (ni+1, nj, nk); v: (0, 0.5, 0); w: (0, 0, 0.5))
__device__ __forceinline__ void mac_f(const float* __restrict__ u, const float* __restrict__ v,
                                      const float* __restrict__ w, int ni, int nj, int nk, float ih, float x, float y,
                                      float z, float& a, float& b, float& c) {
  const AxisF xu = axis_f(x, ih, 0.5f, ni + 1), xvw = axis_f(x, ih, 0.0f, ni);
  const AxisF yv = axis_f(y, ih, 0.5f, nj + 1), yuw = axis_f(y, ih, 0.0f, nj);
  const AxisF zw = axis_f(z, ih, 0.5f, nk + 1), zuv = axis_f(z, ih, 0.0f, nk);
  a = tri_f(u, ni + 1, (ni + 1) * nj, xu, yuw, zuv);
  b = tri_f(v, ni, ni * (nj + 1), xvw, yv, zuv);
  c = tri_f(w, ni, ni * nj, xvw, yuw, zw);
}

// node_world's coordinates without the integer division: the block's run of
// nodes is walked with (i, j, k) carried along
__global__ void advect_rk2_f_kernel(const float* __restrict__ u, const float* __restrict__ v,
                                    const float* __restrict__ w, int ni, int nj, int nk, float ih, GridView f,
                                    GridF ff, float* __restrict__ out, GridF ff2, float* __restrict__ out2, float h,
                                    float dt, int per_block) {
  const size_t n = (size_t)f.nx * f.ny * f.nz;
  const size_t stride = blockDim.x;
  const size_t beg = (size_t)blockIdx.x * per_block;
  const size_t end = beg + per_block < n ? beg + per_block : n;
  const float hf = 0.5f * dt;
  for (size_t e0 = beg + threadIdx.x; e0 < end; e0 += 2 * stride) {
    const size_t e1 = e0 + stride;
    const bool two = e1 < end;
    float wx0, wy0, wz0, wx1 = 0, wy1 = 0, wz1 = 0;
    node_world(f, e0, h, wx0, wy0, wz0);
    if (two) node_world(f, e1, h, wx1, wy1, wz1);
    float a0, b0, c0, a1 = 0, b1 = 0, c1 = 0;
    mac_f(u, v, w, ni, nj, nk, ih, wx0, wy0, wz0, a0, b0, c0);
    if (two) mac_f(u, v, w, ni, nj, nk, ih, wx1, wy1, wz1, a1, b1, c1);
    float px0 = wx0 - hf * a0, py0 = wy0 - hf * b0, pz0 = wz0 - hf * c0;
    float px1 = wx1 - hf * a1, py1 = wy1 - hf * b1, pz1 = wz1 - hf * c1;
    mac_f(u, v, w, ni, nj, nk, ih, px0, py0, pz0, a0, b0, c0);
    if (two) mac_f(u, v, w, ni, nj, nk, ih, px1, py1, pz1, a1, b1, c1);
    px0 = wx0 - dt * a0;
    py0 = wy0 - dt * b0;
    pz0 = wz0 - dt * c0;
    px1 = wx1 - dt * a1;
    py1 = wy1 - dt * b1;
    pz1 = wz1 - dt * c1;
    out[e0] = grid_f(ff, ih, px0, py0, pz0);
    if (out2) out2[e0] = grid_f(ff2, ih, px0, py0, pz0);
    if (two) {
      out[e1] = grid_f(ff, ih, px1, py1, pz1);
      if (out2) out2[e1] = grid_f(ff2, ih, px1, py1, pz1);
    }
  }
}

// ---- the FP32 form again (the same values), specialised to lattice nodes
// when h is a power of two.  A node of the u, v, w or cell-centre lattice
// sits at whole or half-cell coordinates of every MAC velocity grid, so the
// backtrace's first stage (the velocity at the node itself) has axis
// fractions of exactly 0 or 1/2: along an axis where the node and the
// sampled component share their staggering the fraction is 0 and the lerp
// keeps its first corner (lerp_f(a, b, 0) == a for finite values; only the
// sign of a zero can differ, and a zero velocity's sign cannot change
// x - (dt/2) a); where they differ the fraction is 1/2 and the corners are
// (i, i+1) for a staggered component at an unstaggered node, or
// (clamp(i-1), clamp(i)) the other way round.  That stage then reads 9
// values (u-, v-, w-faces) or 6 (cell centres) instead of 24, with no
// coordinate transform; the node's world position is formed in float
// ((i - o) h is exact for a power-of-two h), and node indices are carried
// along the block's run instead of divided out.  The midpoint and final
// samples are advect_rk2_f_kernel's, so outputs are bit for bit its own.

// sampled component C at a node of lattice G (0..2: u, v, w faces, 3: cell
// centres), along axis A: 0 = same staggering, 1 = (i, i+1), 2 = (i-1, i)
__host__ __device__ constexpr int node_axis_mode(int C, int A, int G) {
  return (C == A && G != A) ? 1 : ((C != A && G == A) ? 2 : 0);
}

template <int M>
__device__ __forceinline__ void node_pair(int i, int n, int& a, int& b) {
  if (M == 2) {
    a = i > 0 ? i - 1 : 0;
    b = i < n - 1 ? i : n - 1;
  } else {
    a = i;
    b = i + 1;
  }
}

// component C (extent ni+[C==0], nj+[C==1], nk+[C==2]) at node (i,j,k) of G
template <int C, int G>
__device__ __forceinline__ float node_velocity(const float* __restrict__ d, int ni, int nj, int nk, int i, int j,
                                               int k) {
  constexpr int MX = node_axis_mode(C, 0, G), MY = node_axis_mode(C, 1, G), MZ = node_axis_mode(C, 2, G);
  const int nx = ni + (C == 0), ny = nj + (C == 1), nz = nk + (C == 2);
  const int sy = nx, sz = nx * ny;
  int i0, i1, j0, j1, k0, k1;
  node_pair<MX>(i, nx, i0, i1);
  node_pair<MY>(j, ny, j0, j1);
  node_pair<MZ>(k, nz, k0, k1);
  j0 *= sy;
  j1 *= sy;
  k0 *= sz;
  k1 *= sz;
  auto X = [&](int jk) -> float {
    if constexpr (MX == 0) return __ldg(d + (i0 + jk));
    else return lerp_f(__ldg(d + (i0 + jk)), __ldg(d + (i1 + jk)), 0.5f);
  };
  auto Y = [&](int kk) -> float {
    if constexpr (MY == 0) return X(j0 + kk);
    else return lerp_f(X(j0 + kk), X(j1 + kk), 0.5f);
  };
  if constexpr (MZ == 0) return Y(k0);
  else return lerp_f(Y(k0), Y(k1), 0.5f);
}

__device__ __forceinline__ void node_advance(int& i, int& j, int& k, int by, int nx, int ny) {
  i += by;
  while (i >= nx) {
    i -= nx;
    if (++j == ny) {
      j = 0;
      ++k;
    }
  }
}

struct NodeJob {
  const float* f;  // field on lattice G and its output
  float* out;
  const float* f2;  // optional second field on the same lattice (nullptr: none)
  float* out2;
};

struct NodeJobs {
  NodeJob j[3];
};

template <int G>
__device__ __forceinline__ void advect_nodes(const float* __restrict__ u, const float* __restrict__ v,
                                             const float* __restrict__ w, int ni, int nj, int nk, float ih, float h,
                                             float dt, const NodeJob& job, unsigned blk, int per_block) {
  const int nx = ni + (G == 0), ny = nj + (G == 1), nz = nk + (G == 2);
  const float ox = G == 0 ? 0.5f : 0.0f, oy = G == 1 ? 0.5f : 0.0f, oz = G == 2 ? 0.5f : 0.0f;
  const GridF ff{job.f, nx, ny, nz, ox, oy, oz}, ff2{job.f2, nx, ny, nz, ox, oy, oz};
  float* __restrict__ out = job.out;
  float* __restrict__ out2 = job.out2;
  const size_t n = (size_t)nx * ny * nz;
  const int stride = blockDim.x;
  const size_t beg = (size_t)blk * per_block;
  if (beg >= n) return;
  const size_t end = beg + per_block < n ? beg + per_block : n;
  const float hf = 0.5f * dt;
  int i, j, k;
  decode3(beg + threadIdx.x, nx, ny, i, j, k);
  for (size_t e0 = beg + threadIdx.x; e0 < end; e0 += 2 * (size_t)stride) {
    const size_t e1 = e0 + stride;
    const bool two = e1 < end;
    int i1 = i, j1 = j, k1 = k;
    node_advance(i1, j1, k1, stride, nx, ny);
    const float wx0 = ((float)i - ox) * h, wy0 = ((float)j - oy) * h, wz0 = ((float)k - oz) * h;
    const float wx1 = two ? ((float)i1 - ox) * h : 0.0f, wy1 = two ? ((float)j1 - oy) * h : 0.0f,
                wz1 = two ? ((float)k1 - oz) * h : 0.0f;
    float a0 = node_velocity<0, G>(u, ni, nj, nk, i, j, k), b0 = node_velocity<1, G>(v, ni, nj, nk, i, j, k),
          c0 = node_velocity<2, G>(w, ni, nj, nk, i, j, k);
    float a1 = 0, b1 = 0, c1 = 0;
    if (two) {
      a1 = node_velocity<0, G>(u, ni, nj, nk, i1, j1, k1);
      b1 = node_velocity<1, G>(v, ni, nj, nk, i1, j1, k1);
      c1 = node_velocity<2, G>(w, ni, nj, nk, i1, j1, k1);
    }
    float px0 = wx0 - hf * a0, py0 = wy0 - hf * b0, pz0 = wz0 - hf * c0;
    float px1 = wx1 - hf * a1, py1 = wy1 - hf * b1, pz1 = wz1 - hf * c1;
    mac_f(u, v, w, ni, nj, nk, ih, px0, py0, pz0, a0, b0, c0);
    if (two) mac_f(u, v, w, ni, nj, nk, ih, px1, py1, pz1, a1, b1, c1);
    px0 = wx0 - dt * a0;
    py0 = wy0 - dt * b0;
    pz0 = wz0 - dt * c0;
    px1 = wx1 - dt * a1;
    py1 = wy1 - dt * b1;
    pz1 = wz1 - dt * c1;
    out[e0] = grid_f(ff, ih, px0, py0, pz0);
    if (out2) out2[e0] = grid_f(ff2, ih, px0, py0, pz0);
    if (two) {
      out[e1] = grid_f(ff, ih, px1, py1, pz1);
      if (out2) out2[e1] = grid_f(ff2, ih, px1, py1, pz1);
    }
    i = i1;
    j = j1;
    k = k1;
    node_advance(i, j, k, stride, nx, ny);
  }
}

// Block b runs job b % njobs on run b / njobs of its lattice, g0 + job (one
// launch advects u, v and w with g0 = 0 and three jobs, or one lattice's
// field or field pair with a single job).  Interleaving the jobs block by
// block keeps the three components' blocks in flight over the same region,
// so the velocity they all sample is read from DRAM about once.
__global__ void __launch_bounds__(256) advect_rk2_node_kernel(const float* __restrict__ u,
                                                              const float* __restrict__ v,
                                                              const float* __restrict__ w, int ni, int nj, int nk,
                                                              float ih, float h, float dt, NodeJobs jobs, int g0,
                                                              int njobs, int per_block) {
  const unsigned q = blockIdx.x % (unsigned)njobs, blk = blockIdx.x / (unsigned)njobs;
  const NodeJob job = q == 0 ? jobs.j[0] : (q == 1 ? jobs.j[1] : jobs.j[2]);
  switch (g0 + (int)q) {
    case 0: advect_nodes<0>(u, v, w, ni, nj, nk, ih, h, dt, job, blk, per_block); break;
    case 1: advect_nodes<1>(u, v, w, ni, nj, nk, ih, h, dt, job, blk, per_block); break;
    case 2: advect_nodes<2>(u, v, w, ni, nj, nk, ih, h, dt, job, blk, per_block); break;
    default: advect_nodes<3>(u, v, w, ni, nj, nk, ih, h, dt, job, blk, per_block); break;
  }
}

// getDelta, Smoke_solver3D.cpp:1298-1319
__global__ void delta_kernel(const float* __restrict__ after, const float* __restrict__ before,
                             float* __restrict__ delta, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    delta[e] = after[e] - before[e];
}

// ------------------------------------------------------------------ P2G
// The reference's particle record (fluid_particle.h:14-20), 40 bytes.
struct ParticleRec {
  float pos[3];
  float vel[3];
  float dens, temp;
  int hash_idx, sub_hash_idx;
};
static_assert(sizeof(ParticleRec) == 40, "particle record is 40 bytes");

// hash_FLIP cell, Smoke_solver3D.cpp:1337-1343: int((pos + 0.5h)/h) with
// C truncation; values outside (-1, n) (and NaN) are out of range, as the
// x86 conversion makes them in the reference.
// x / h in float, exactly as IEEE division; a multiplication when h is a
// power of two (inv_h != 0), which is then exact
__device__ __forceinline__ float fdiv_h(float x, float h, float inv_h) { return inv_h != 0.0f ? x * inv_h : x / h; }

__device__ __forceinline__ int hash_cell(const float* pos, int ni, int nj, int nk, float h, float inv_h) {
  const float c = 0.5f * h;
  float tx = fdiv_h(pos[0] + c, h, inv_h), ty = fdiv_h(pos[1] + c, h, inv_h), tz = fdiv_h(pos[2] + c, h, inv_h);
  if (!(tx > -1.0f && tx < (float)ni)) return -1;
  if (!(ty > -1.0f && ty < (float)nj)) return -1;
  if (!(tz > -1.0f && tz < (float)nk)) return -1;
  return ((int)tz * nj + (int)ty) * ni + (int)tx;
}

// The frame of a nested subdomain grid (SubDomainSolver): origin bmin in
// world space; `sub` selects its clamped hash.  The main grid passes origin 0
// and sub = 0 (x - 0.0f is x, so its arithmetic is unchanged).
struct SubFrame {
  float bx, by, bz;
  int sub;
};

// SubDomainSolver::hash_FLIP, sub_domain.cpp:1087-1109: the cell of
// pos - bmin + h/2, truncated (x86 semantics: out of range or NaN gives
// INT_MIN) and clamped into the grid, so every particle is hashed.
__device__ __forceinline__ int trunc_x86(float t) {
  return (t >= -2147483648.0f && t < 2147483648.0f) ? (int)t : INT_MIN;
}
__device__ __forceinline__ int sub_hash_cell(const float* pos, int ni, int nj, int nk, float h, float inv_h,
                                             const SubFrame& f) {
  const float b[3] = {f.bx, f.by, f.bz};
  const int n[3] = {ni, nj, nk};
  int c[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float x = pos[a] - b[a];
    x = x + 0.5f * h;
    const int t = trunc_x86(fdiv_h(x, h, inv_h));
    c[a] = t < 0 ? 0 : (t > n[a] - 1 ? n[a] - 1 : t);
  }
  return (c[2] * nj + c[1]) * ni + c[0];
}

__global__ void hash_count_kernel(const ParticleRec* __restrict__ p, int np, int ni, int nj, int nk, float h,
                                  float inv_h, int* __restrict__ cell, int* __restrict__ slot,
                                  int* __restrict__ count, SubFrame sf) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
    int c = sf.sub ? sub_hash_cell(p[q].pos, ni, nj, nk, h, inv_h, sf) : hash_cell(p[q].pos, ni, nj, nk, h, inv_h);
    cell[q] = c;
    // the lanes of a warp that share a cell take consecutive slots in lane
    // (particle) order with one atomic, so a bucket is a few runs of
    // consecutive particle indices where the particles come in cell order
    const unsigned grp = __match_any_sync(__activemask(), c);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    int base = 0;
    if (lane == leader && c >= 0) base = atomicAdd(count + c, __popc(grp));
    base = __shfl_sync(grp, base, leader);
    slot[q] = (c >= 0) ? base + __popc(grp & ((1u << lane) - 1u)) : -1;
  }
}

// Exclusive scan of int counts, three-phase (block scan, scan of block
// sums, add).  SCAN_BLOCK threads x 4 items per block.
constexpr int kScanBlock = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sm, int& total) {
  // warp inclusive
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = (lane < kScanBlock / 32) ? sm[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanBlock / 32) sm[lane] = s;
  }
  __syncthreads();
  int warp_prefix = (wid > 0) ? sm[wid - 1] : 0;
  total = sm[kScanBlock / 32 - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

__global__ void __launch_bounds__(kScanBlock) scan_tiles_kernel(const int* __restrict__ in, int* __restrict__ out,
                                                               int* __restrict__ tile_sums, size_t n) {
  __shared__ int sm[32];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int local = 0;
#pragma unroll
  for (int t = 0; t < kScanItems; ++t) {
    v[t] = (base + t < n) ? in[base + t] : 0;
    local += v[t];
  }
  int total;
  int pre = block_exclusive_scan(local, sm, total);
#pragma unroll
  for (int t = 0; t < kScanItems; ++t) {
    if (base + t < n) out[base + t] = pre;
    pre += v[t];
  }
  if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

__global__ void scan_add_kernel(int* __restrict__ out, const int* __restrict__ tile_prefix, size_t n) {
  size_t base = (size_t)blockIdx.x * kScanTile;
  int add = tile_prefix[blockIdx.x];
  for (int t = threadIdx.x; t < kScanTile; t += blockDim.x)
    if (base + t < n) out[base + t] += add;
}

__global__ void scatter_kernel(const int* __restrict__ cell, const int* __restrict__ slot,
                               const int* __restrict__ start, int* __restrict__ order, int np) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
    int c = cell[q];
    if (c >= 0) order[start[c] + slot[q]] = q;
  }
}

// Put every bucket into ascending particle order (the order hash_FLIP
// pushes them in).  Insertion sort for the usual handful of particles per
// cell, heapsort beyond 32.
__device__ __forceinline__ void sift_down(int* a, int root, int end) {
  while (true) {
    int child = 2 * root + 1;
    if (child >= end) return;
    if (child + 1 < end && a[child] < a[child + 1]) ++child;
    if (a[root] >= a[child]) return;
    int t = a[root]; a[root] = a[child]; a[child] = t;
    root = child;
  }
}

// Buckets of 33 .. kBigBucket particles are listed in `big` (big_n counts
// them) for sort_big_buckets_kernel; larger ones are heapsorted here.
constexpr int kBigBucket = 2048;

__global__ void sort_buckets_kernel(const int* __restrict__ start, int* __restrict__ order, int ncells,
                                    int* __restrict__ big, int* __restrict__ big_n) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
    int b = start[c], e = start[c + 1];
    int m = e - b;
    if (m < 2) continue;
    int* a = order + b;
    if (m > 32 && m <= kBigBucket) {
      big[atomicAdd(big_n, 1)] = c;
      continue;
    }
    if (m <= 32) {
      for (int x = 1; x < m; ++x) {
        int key = a[x];
        int y = x - 1;
        while (y >= 0 && a[y] > key) { a[y + 1] = a[y]; --y; }
        a[y + 1] = key;
      }
    } else {
      for (int r = m / 2 - 1; r >= 0; --r) sift_down(a, r, m);
      for (int end = m - 1; end > 0; --end) {
        int t = a[0]; a[0] = a[end]; a[end] = t;
        sift_down(a, 0, end);
      }
    }
  }
}

// Bitonic sort (ascending) of P keys in shared memory by one warp, P a
// power of two >= 32; `pay`, when given, moves with the keys.  Within a
// stage the compare-exchange pairs are disjoint; the warp synchronises
// between stages.
__device__ __forceinline__ void warp_bitonic(int* key, int* pay, int P, int lane) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < P; i += 32) {
        const int x = i ^ j;
        if (x > i) {
          const int p = key[i], q = key[x];
          if ((p > q) == ((i & k) == 0)) {
            key[i] = q;
            key[x] = p;
            if (pay) {
              const int t = pay[i];
              pay[i] = pay[x];
              pay[x] = t;
            }
          }
        }
      }
      __syncwarp();
    }
  }
}

// The listed buckets, one warp each, into ascending particle order.  A
// bucket is read as runs of consecutive particle indices (hash_count_kernel
// gives a warp's particles of one cell consecutive slots, so particles that
// come in cell order leave few runs); the runs are disjoint integer ranges,
// so the bucket in order is the runs sorted by their first index and
// written out as ranges.  A bucket of more than kBigRuns runs is sorted by
// a least-significant-digit radix sort of (index - the bucket's smallest)
// in 8-bit digits, as many passes as that range needs: per pass a
// shared-memory histogram, its scan, and a stable scatter of 32 entries at
// a time in order (each entry's rank among the earlier equal digits of its
// 32 from __match_any_sync).  Particle indices are distinct, so either
// gives the order the heapsort gives.
constexpr int kBigWarps = 2;
constexpr int kBigRuns = 128;

__global__ void __launch_bounds__(32 * kBigWarps) sort_big_buckets_kernel(const int* __restrict__ start,
                                                                       int* __restrict__ order,
                                                                       const int* __restrict__ big,
                                                                       const int* __restrict__ big_n) {
  __shared__ int sm[kBigWarps][2][kBigBucket];
  __shared__ int hist[kBigWarps][256];
  __shared__ int rkey[kBigWarps][kBigRuns], rlen[kBigWarps][kBigRuns];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int *v = sm[wid][0], *u = sm[wid][1], *cnt = hist[wid], *rk = rkey[wid], *rl = rlen[wid];
  const int nbig = *big_n;
  for (int e = blockIdx.x * kBigWarps + wid; e < nbig; e += gridDim.x * kBigWarps) {
    const int c = big[e];
    const int b = start[c], m = start[c + 1] - b;
    int lo = INT_MAX, hi = 0;
    for (int i = lane; i < m; i += 32) {
      const int x = order[b + i];
      v[i] = x;
      lo = min(lo, x);
      hi = max(hi, x);
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __syncwarp();
    // run heads: position x starts a run unless v[x] == v[x - 1] + 1
    int nrun = 0;
    for (int x0 = 0; x0 < m; x0 += 32) {
      const int x = x0 + lane;
      const bool head = x < m && (x == 0 || v[x] != v[x - 1] + 1);
      const unsigned hm = __ballot_sync(0xffffffffu, head);
      const int idx = nrun + __popc(hm & lt);
      if (head && idx < kBigRuns) rk[idx] = x;
      nrun += __popc(hm);
    }
    __syncwarp();
    if (nrun <= kBigRuns) {
      for (int r = lane; r < nrun; r += 32) rl[r] = (r + 1 < nrun ? rk[r + 1] : m) - rk[r];
      __syncwarp();
      int P = 32;
      while (P < nrun) P <<= 1;
      for (int r = lane; r < P; r += 32) {
        if (r < nrun) {
          rk[r] = v[rk[r]];
        } else {
          rk[r] = INT_MAX;
          rl[r] = 0;
        }
      }
      __syncwarp();
      warp_bitonic(rk, rl, P, lane);
      int off = 0;
      for (int r = 0; r < nrun; ++r) {
        const int k0 = rk[r], len = rl[r];
        for (int x = lane; x < len; x += 32) order[b + off + x] = k0 + x;
        off += len;
      }
    } else {
      const unsigned span = (unsigned)(hi - lo);
      for (int shift = 0; shift == 0 || (shift < 32 && (span >> shift) != 0u); shift += 8) {
        for (int d = lane; d < 256; d += 32) cnt[d] = 0;
        __syncwarp();
        for (int i = lane; i < m; i += 32) atomicAdd(cnt + ((unsigned)(v[i] - lo) >> shift & 255u), 1);
        __syncwarp();
        {  // exclusive scan of the 256 counts, 8 consecutive bins per lane
          int t[8], sum = 0;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            t[q] = cnt[8 * lane + q];
            sum += t[q];
          }
          int x = sum;
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
          }
          int pre = x - sum;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            cnt[8 * lane + q] = pre;
            pre += t[q];
          }
        }
        __syncwarp();
        for (int x0 = 0; x0 < m; x0 += 32) {
          const int x = x0 + lane;
          const bool ok = x < m;
          const int val = ok ? v[x] : 0;
          const int d = ok ? (int)((unsigned)(val - lo) >> shift & 255u) : 256;
          const unsigned peers = __match_any_sync(0xffffffffu, d);
          const int base = ok ? cnt[d] : 0;
          if (ok) u[base + __popc(peers & lt)] = val;
          __syncwarp();
          if (ok && (peers & lt) == 0u) cnt[d] = base + __popc(peers);
          __syncwarp();
        }
        int* w = v;
        v = u;
        u = w;
      }
      for (int i = lane; i < m; i += 32) order[b + i] = v[i];
      v = sm[wid][0];
      u = sm[wid][1];
    }
    __syncwarp();
  }
}

// Sorted structure-of-arrays copy for the gather: pos.xyz + a flag in .w
// (1 when all three velocity components are finite), vel.xyz.
// Only the start[ncells] bucketed particles are gathered (`total` points at
// that count on the device); particles outside the grid have no slot.
// Positions are relative to the grid's origin (pos - bmin).
__global__ void gather_sorted_kernel(const ParticleRec* __restrict__ p, const int* __restrict__ order,
                                     float4* __restrict__ spos, float4* __restrict__ svel,
                                     const int* __restrict__ total, SubFrame sf) {
  const int nsorted = *total;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nsorted; e += gridDim.x * blockDim.x) {
    const ParticleRec& r = p[order[e]];
    bool fin = isfinite(r.vel[0]) && isfinite(r.vel[1]) && isfinite(r.vel[2]);
    spos[e] = make_float4(r.pos[0] - sf.bx, r.pos[1] - sf.by, r.pos[2] - sf.bz, fin ? 1.0f : 0.0f);
    svel[e] = make_float4(r.vel[0], r.vel[1], r.vel[2], 0.0f);
  }
}

// SmokeSolver3D::H, Smoke_solver3D.h:217-223: 1 + r on [-1, 0), 1 - r on
// [0, 1), else 0 (NaN included).  Written as max(1 - |r|, 0): on [-1, 0)
// 1 - (-r) is the same rounded sum as 1 + r; for |r| >= 1 (and r = +-inf)
// 1 - |r| <= 0 and the maximum is +0; fmaxf returns 0 for a NaN r.
__device__ __forceinline__ float tent(float r) { return fmaxf(1.0f - fabsf(r), 0.0f); }

// particle_to_grid, Smoke_solver3D.cpp:1451-1510, for the three velocity
// components in one pass: at each face node, field = sum(w v)/sum(w),
// coef = sum(w), sum(w) starting at 1e-5, weight H(dx/h)H(dy/h)H(dz/h).  One
// thread takes index (i, j, k) of all three face grids (u: (ni+1) x nj x nk,
// v: ni x (nj+1) x nk, w: ni x nj x (nk+1); a component whose output is null
// or whose grid does not hold (i, j, k) is skipped): the three nodes gather
// from the same buckets in the same order and share their offsets pairwise,
// so each particle is loaded once, six one-dimensional tents give the three
// weights, and every component's sums are those of its own pass, bit for bit.  A
// particle whose offset from a node exceeds 1.0001 h on some axis has weight
// exactly 0 and (finite velocity) contributes exactly nothing to that node,
// so it is skipped there without changing any sum.
// SUB: SubDomainSolver::particle_to_grid (sub_domain.cpp:1204-1265) with
// determineDist (sub_domain.h:89-103): within 4 cells of the grid's boundary
// the tent is 4h wide over the 9^3 neighbouring buckets.
//
// `part` picks the nodes a launch takes: P2G_ALL every index; for a
// subdomain P2G_SHELL the indices within 4 of the boundary on some axis
// (the 9^3 gathers) and P2G_INNER the box between, so that no warp mixes the
// two costs.  The shell is enumerated as the end planes (k), then the end
// rows (j) of the inner planes, then the end nodes (i) of the inner rows;
// per axis the inner range is [5, n - 5] (m = max(0, n - 9) indices) and an
// end index t in [0, n + 1 - m) is t below 5, else t + m.
enum { P2G_ALL = 0, P2G_INNER = 1, P2G_SHELL = 2 };

__host__ __device__ inline size_t p2g_part_size(int part, int ni, int nj, int nk) {
  const size_t X = (size_t)ni + 1, Y = (size_t)nj + 1, Z = (size_t)nk + 1;
  const size_t mi = ni > 9 ? ni - 9 : 0, mj = nj > 9 ? nj - 9 : 0, mk = nk > 9 ? nk - 9 : 0;
  if (part == P2G_ALL) return X * Y * Z;
  if (part == P2G_INNER) return mi * mj * mk;
  return (Z - mk) * X * Y + mk * (Y - mj) * X + mk * mj * (X - mi);
}

// The face-node triple (i, j, k) of the u, v, w grids during a gather:
// node coordinates, which components it holds, and the running sums.
struct P2gNode {
  float xi, xh, yj, yh, zk, zh;
  bool act0, act1, act2;
  float tw[3], tv[3];
};

__device__ __forceinline__ P2gNode p2g_node(int i, int j, int k, int ni, int nj, int nk, float h, bool hu, bool hv,
                                            bool hw) {
  P2gNode n;
  n.act0 = hu && j < nj && k < nk;
  n.act1 = hv && i < ni && k < nk;
  n.act2 = hw && i < ni && j < nj;
  // node positions: the component's own axis sits half a cell lower
  n.xi = (float)((double)(float)i * (double)h);
  n.xh = (float)(((double)(float)i - 0.5) * (double)h);
  n.yj = (float)((double)(float)j * (double)h);
  n.yh = (float)(((double)(float)j - 0.5) * (double)h);
  n.zk = (float)((double)(float)k * (double)h);
  n.zh = (float)(((double)(float)k - 0.5) * (double)h);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    n.tw[c] = 1e-5f;
    n.tv[c] = 0.0f;
  }
  return n;
}

// One particle's step of the gather at node n: the particle at (px, py, pz)
// (grid-relative), `fin` when its velocity is finite; `vel()` fetches the
// velocity, called only when some component takes the particle.  The nodes
// share offsets pairwise (x of v and w, y of u and w, z of u and v): six
// one-dimensional tents serve the three weights.
template <typename VelF>
__device__ __forceinline__ void p2g_visit(P2gNode& n, float px, float py, float pz, bool fin, float hk, float ihk,
                                          float rk, VelF vel) {
  const float dxu = px - n.xh, dxv = px - n.xi;
  const float dyu = py - n.yj, dyv = py - n.yh;
  const float dzu = pz - n.zk, dzw = pz - n.zh;
  const bool ox = fabsf(dxu) >= rk, oxv = fabsf(dxv) >= rk, oy = fabsf(dyu) >= rk, oyv = fabsf(dyv) >= rk;
  const bool oz = fabsf(dzu) >= rk, ozw = fabsf(dzw) >= rk;
  const bool ok0 = n.act0 && !(fin && (ox || oy || oz));
  const bool ok1 = n.act1 && !(fin && (oxv || oyv || oz));
  const bool ok2 = n.act2 && !(fin && (oxv || oy || ozw));
  if (!(ok0 || ok1 || ok2)) return;
  const float txu = tent(fdiv_h(dxu, hk, ihk)), txv = tent(fdiv_h(dxv, hk, ihk));
  const float tyu = tent(fdiv_h(dyu, hk, ihk)), tyv = tent(fdiv_h(dyv, hk, ihk));
  const float tzu = tent(fdiv_h(dzu, hk, ihk)), tzw = tent(fdiv_h(dzw, hk, ihk));
  const float3 vv = vel();
  if (ok0) {
    const float wgt = txu * tyu * tzu;
    n.tw[0] = n.tw[0] + wgt;
    n.tv[0] = n.tv[0] + wgt * vv.x;
  }
  if (ok1) {
    const float wgt = txv * tyv * tzu;
    n.tw[1] = n.tw[1] + wgt;
    n.tv[1] = n.tv[1] + wgt * vv.y;
  }
  if (ok2) {
    const float wgt = txv * tyu * tzw;
    n.tw[2] = n.tw[2] + wgt;
    n.tv[2] = n.tv[2] + wgt * vv.z;
  }
}

// The tent of an offset d from a node, in units of h.  M = 0: d / h; M = 1:
// h a power of two, d * inv_h (exact); M = 2: h a power of two <= 1 and the
// positions and node coordinates already multiplied by inv_h: scaling by a
// power of two >= 1 is exact and commutes with the rounded difference, so d
// is the scaled offset itself (an overflow to inf gives tent 0 either way).
template <int M>
__device__ __forceinline__ float p2g_tent(float d, float h, float inv_h) {
  return tent(M == 0 ? d / h : (M == 1 ? d * inv_h : d));
}

// One particle of node n's window added as the reference's loop adds it,
// with no reach test: a particle out of reach has weight exactly 0 and adds
// +0 to sum(w) and +-0 to sum(w v) (which never holds -0), so the sums are
// those of p2g_visit; a non-finite velocity makes sum(w v) NaN in both.
// Inactive components are summed and not stored.
template <int M>
__device__ __forceinline__ void p2g_add(P2gNode& n, float px, float py, float pz, float vx, float vy, float vz,
                                        float h, float inv_h) {
  const float txu = p2g_tent<M>(px - n.xh, h, inv_h), txv = p2g_tent<M>(px - n.xi, h, inv_h);
  const float tyu = p2g_tent<M>(py - n.yj, h, inv_h), tyv = p2g_tent<M>(py - n.yh, h, inv_h);
  const float tzu = p2g_tent<M>(pz - n.zk, h, inv_h), tzw = p2g_tent<M>(pz - n.zh, h, inv_h);
  const float w0 = txu * tyu * tzu, w1 = txv * tyv * tzu, w2 = txv * tyu * tzw;
  n.tw[0] = n.tw[0] + w0;
  n.tv[0] = n.tv[0] + w0 * vx;
  n.tw[1] = n.tw[1] + w1;
  n.tv[1] = n.tv[1] + w1 * vy;
  n.tw[2] = n.tw[2] + w2;
  n.tv[2] = n.tv[2] + w2 * vz;
}

// p2g_add for the nodes (i, j, k) and (i, j, k + 1) at once: they share the
// x and y tents and the products tx * ty, so each weight is the same
// product as p2g_add forms, with the node's own z tent.
template <int M>
__device__ __forceinline__ void p2g_add2(P2gNode& a, P2gNode& b, float px, float py, float pz, float vx, float vy,
                                         float vz, float h, float inv_h) {
  const float txu = p2g_tent<M>(px - a.xh, h, inv_h), txv = p2g_tent<M>(px - a.xi, h, inv_h);
  const float tyu = p2g_tent<M>(py - a.yj, h, inv_h), tyv = p2g_tent<M>(py - a.yh, h, inv_h);
  const float uu = txu * tyu, vv = txv * tyv, ww = txv * tyu;
  const float tzua = p2g_tent<M>(pz - a.zk, h, inv_h), tzwa = p2g_tent<M>(pz - a.zh, h, inv_h);
  const float tzub = p2g_tent<M>(pz - b.zk, h, inv_h), tzwb = p2g_tent<M>(pz - b.zh, h, inv_h);
  const float a0 = uu * tzua, a1 = vv * tzua, a2 = ww * tzwa;
  const float b0 = uu * tzub, b1 = vv * tzub, b2 = ww * tzwb;
  a.tw[0] = a.tw[0] + a0;
  a.tv[0] = a.tv[0] + a0 * vx;
  a.tw[1] = a.tw[1] + a1;
  a.tv[1] = a.tv[1] + a1 * vy;
  a.tw[2] = a.tw[2] + a2;
  a.tv[2] = a.tv[2] + a2 * vz;
  b.tw[0] = b.tw[0] + b0;
  b.tv[0] = b.tv[0] + b0 * vx;
  b.tw[1] = b.tw[1] + b1;
  b.tv[1] = b.tv[1] + b1 * vy;
  b.tw[2] = b.tw[2] + b2;
  b.tv[2] = b.tv[2] + b2 * vz;
}

// field = sum(w v) / sum(w), coef = sum(w) at the components node n holds
__device__ __forceinline__ void p2g_store(const P2gNode& n, int i, int j, int k, int ni, int nj, float* fu,
                                          float* cu, float* fv, float* cv, float* fw, float* cw) {
  if (n.act0) {
    const size_t o = (size_t)i + (size_t)(ni + 1) * ((size_t)j + (size_t)nj * k);
    cu[o] = n.tw[0];
    fu[o] = n.tv[0] / n.tw[0];
  }
  if (n.act1) {
    const size_t o = (size_t)i + (size_t)ni * ((size_t)j + (size_t)(nj + 1) * k);
    cv[o] = n.tw[1];
    fv[o] = n.tv[1] / n.tw[1];
  }
  if (n.act2) {
    const size_t o = (size_t)i + (size_t)ni * ((size_t)j + (size_t)nj * k);
    cw[o] = n.tw[2];
    fw[o] = n.tv[2] / n.tw[2];
  }
}

// The gather of node n from the global sorted arrays: the buckets i-l..i+l
// of each row (ck, cj) of the (2l+1)^2 neighbouring rows, rows in order of
// k then j, each row's buckets one consecutive run of particles in the
// sorted order, visited in that order.
__device__ __forceinline__ void p2g_gather_global(P2gNode& n, int i, int j, int k, int l, int ni, int nj, int nk,
                                                  float hk, float ihk, float rk, const int* __restrict__ start,
                                                  const float4* __restrict__ spos,
                                                  const float4* __restrict__ svel) {
  for (int dk = -l; dk <= l; ++dk) {
    const int ck = k + dk;
    if (ck < 0 || ck >= nk) continue;
    for (int dj = -l; dj <= l; ++dj) {
      const int cj = j + dj;
      if (cj < 0 || cj >= nj) continue;
      const int row = (ck * nj + cj) * ni;
      const int b = __ldg(start + row + max(i - l, 0)), en = __ldg(start + row + min(i + l, ni - 1) + 1);
      for (int q = b; q < en; ++q) {
        const float4 pp = __ldg(spos + q);
        p2g_visit(n, pp.x, pp.y, pp.z, pp.w != 0.0f, hk, ihk, rk, [&] {
          const float4 vv = __ldg(svel + q);
          return make_float3(vv.x, vv.y, vv.z);
        });
      }
    }
  }
}

template <bool SUB>
__global__ void p2g3_kernel(const int* __restrict__ start, const float4* __restrict__ spos,
                            const float4* __restrict__ svel, float* __restrict__ fu, float* __restrict__ cu,
                            float* __restrict__ fv, float* __restrict__ cv, float* __restrict__ fw,
                            float* __restrict__ cw, int ni, int nj, int nk, float h, float inv_h, int part) {
  const size_t n = p2g_part_size(part, ni, nj, nk);
  const int X = ni + 1, Y = nj + 1, Z = nk + 1;
  const int mi = max(ni - 9, 0), mj = max(nj - 9, 0), mk = max(nk - 9, 0);
  const size_t p1 = (size_t)(Z - mk) * X * Y, p2 = (size_t)mk * (Y - mj) * X;
  const float reach = h * 1.0001f;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    if (part == P2G_ALL) {
      decode3(e, X, Y, i, j, k);
    } else if (part == P2G_INNER) {
      decode3(e, mi, mj, i, j, k);
      i += 5;
      j += 5;
      k += 5;
    } else if (e < p1) {  // end planes
      decode3(e, X, Y, i, j, k);
      k = k < 5 ? k : k + mk;
    } else if (e < p1 + p2) {  // end rows of the inner planes
      decode3(e - p1, X, Y - mj, i, j, k);
      j = j < 5 ? j : j + mj;
      k += 5;
    } else {  // end nodes of the inner rows
      decode3(e - p1 - p2, X - mi, mj, i, j, k);
      i = i < 5 ? i : i + mi;
      j += 5;
      k += 5;
    }
    P2gNode nd = p2g_node(i, j, k, ni, nj, nk, h, fu != nullptr, fv != nullptr, fw != nullptr);
    if (!(nd.act0 || nd.act1 || nd.act2)) continue;
    int l = 1;
    float hk = h, ihk = inv_h, rk = reach;
    if (SUB) {
      const int dist = min(min(min(i, ni - i), min(j, nj - j)), min(k, nk - k));
      if (dist <= 4) {
        l = 4;
        hk = (float)(4.0 * (double)h);
        ihk = inv_h * 0.25f;  // exact: inv_h is a power of two or 0
        rk = hk * 1.0001f;
      }
    }
    p2g_gather_global(nd, i, j, k, l, ni, nj, nk, hk, ihk, rk, start, spos, svel);
    p2g_store(nd, i, j, k, ni, nj, fu, cu, fv, cv, fw, cw);
  }
}

// The tiled gather (main grid, every node index): a CTA owns an 8 x 8 x TZ
// tile of face-node indices (i, j, k), two nodes (k, k + 1) per thread, and
// stages the particles its nodes gather from - the buckets of the tile's
// cells and a one-cell ring, each row of them one consecutive run of the
// sorted order - in shared memory, positions and velocities as six float
// arrays; the threads then gather from there.  In the global form each
// thread streams its own runs through L1, the 32 threads of a warp reading
// 32 runs about a bucket apart; here the loads are coalesced once per tile,
// and a thread's two nodes share the x run and the x and y tents of the
// planes both windows hold.  A region holding more than `cap` particles is
// staged in chunks of `cap`: the staged sequence is the row runs in row
// order and a node's window is a sub-run of each of its rows, taken in that
// order, so chunk by chunk each node adds the part of its window the chunk
// holds and its visiting order is unchanged.  Every particle of a window is
// added (p2g_add: no reach test, no divergence between the threads of a
// warp), which gives p2g_visit's sums bit for bit.
// Tile shapes: TZ = 8 node layers (one CTA of 256 threads per SM) or TZ = 4
// (two CTAs of 128 threads per SM, each half the shared memory, so that one
// CTA's staging overlaps the other's gathers).  SUB: a subdomain's grid,
// whose nodes within 4 of its boundary gather from 9^3 buckets: the tables
// hold a 4-cell ring.
constexpr int kP2gTX = 8, kP2gTY = 8;
constexpr int kP2gBatch = 4;  // 32-particle steps a warp loads before staging them
template <int TZ, bool SUB>
struct P2gTile {
  static constexpr int ring = SUB ? 4 : 1;                          // widest window half-width
  static constexpr int threads = kP2gTX * kP2gTY * (TZ / 2);         // two nodes (k, k + 1) per thread
  static constexpr int rx = kP2gTX + 2 * ring;                       // bucket columns of the staged region
  static constexpr int rows = (kP2gTY + 2 * ring) * (TZ + 2 * ring);  // bucket rows of the staged region
  static constexpr int rows_pad = (rows + 1 + 31) / 32 * 32;          // the row scan's width
  static constexpr int fixed_ints = rows * (rx + 1) + 2 * rows_pad;
  static constexpr int ctas_per_sm = TZ == 8 ? 1 : 2;
  static_assert(fixed_ints % 4 == 0, "p2g tile tables");
};

// shared-memory slot of staged particle s: one pad word per 32 spreads the
// reads of neighbouring nodes, about a bucket apart, over the banks
__host__ __device__ inline int p2g_slot(int s) { return s + (s >> 5); }

// particles a CTA with `smem_bytes` of dynamic shared memory stages
template <int TZ, bool SUB>
__host__ __device__ inline int p2g_tile_cap(size_t smem_bytes) {
  const size_t fixed = sizeof(int) * (size_t)P2gTile<TZ, SUB>::fixed_ints;
  if (smem_bytes <= fixed + 6 * sizeof(float) * 2) return 0;
  const long a = (long)((smem_bytes - fixed) / (6 * sizeof(float)));  // floats per array
  long cap = (a - 1) * 32 / 33;
  while (cap > 0 && p2g_slot((int)cap - 1) + 1 > a) --cap;
  return (int)cap;
}

// The staged particles of one chunk and where each row's buckets start.
struct P2gStage {
  const int* cs;  // [row][c]: staged index of bucket clo + c's first particle (row stride `stride`)
  int stride, clo, cjlo, cklo, nry;
  int c0, c1;  // the chunk: staged indices [c0, c1)
  const float *px, *py, *pz, *vx, *vy, *vz;
};

// the window i - l .. i + l (clipped to the grid) of row (ck, cj), clipped
// to the chunk and made chunk-relative
__device__ __forceinline__ int2 p2g_window(const P2gStage& g, int ck, int cj, int i, int l, int ni) {
  const int* c = g.cs + ((ck - g.cklo) * g.nry + (cj - g.cjlo)) * g.stride;
  return make_int2(max(c[max(i - l, 0) - g.clo], g.c0) - g.c0, min(c[min(i + l, ni - 1) + 1 - g.clo], g.c1) - g.c0);
}

template <int M>
__device__ __forceinline__ void p2g_run1(P2gNode& n, int b, int e, const P2gStage& g, float hk, float ihk) {
#pragma unroll 2
  for (int s = b; s < e; ++s) {
    const int P = p2g_slot(s);
    p2g_add<M>(n, g.px[P], g.py[P], g.pz[P], g.vx[P], g.vy[P], g.vz[P], hk, ihk);
  }
}

template <int M>
__device__ __forceinline__ void p2g_run2(P2gNode& n0, P2gNode& n1, int b, int e, const P2gStage& g, float hk,
                                         float ihk) {
#pragma unroll 2
  for (int s = b; s < e; ++s) {
    const int P = p2g_slot(s);
    p2g_add2<M>(n0, n1, g.px[P], g.py[P], g.pz[P], g.vx[P], g.vy[P], g.vz[P], hk, ihk);
  }
}

// One chunk's gathers of the nodes (i, j, k) and (i, j, k + 1), both of
// window half-width l: planes k - l .. k + 1 + l in order, rows j - l ..
// j + l in each; the planes both windows hold are visited once for both
// (the same x run), k - l only by the first node, k + 1 + l only by the
// second.  on1 false: the first node alone.
template <int M>
__device__ __forceinline__ void p2g_chunk2(P2gNode& n0, P2gNode& n1, bool on1, int l, int i, int j, int k, int ni,
                                           int nj, int nk, const P2gStage& g, float hk, float ihk) {
  for (int ck = k - l; ck <= k + 1 + l; ++ck) {
    const bool a0 = ck <= k + l, a1 = on1 && ck >= k + 1 - l;
    if (ck < 0 || ck >= nk || !(a0 || a1)) continue;
    for (int cj = j - l; cj <= j + l; ++cj) {
      if (cj < 0 || cj >= nj) continue;
      const int2 w = p2g_window(g, ck, cj, i, l, ni);
      if (a0 && a1)
        p2g_run2<M>(n0, n1, w.x, w.y, g, hk, ihk);
      else if (a0)
        p2g_run1<M>(n0, w.x, w.y, g, hk, ihk);
      else
        p2g_run1<M>(n1, w.x, w.y, g, hk, ihk);
    }
  }
}

// The same for a single node of half-width l.
template <int M>
__device__ __forceinline__ void p2g_chunk1(P2gNode& n, int l, int i, int j, int k, int ni, int nj, int nk,
                                           const P2gStage& g, float hk, float ihk) {
  for (int ck = max(k - l, 0); ck <= min(k + l, nk - 1); ++ck)
    for (int cj = max(j - l, 0); cj <= min(j + l, nj - 1); ++cj) {
      const int2 w = p2g_window(g, ck, cj, i, l, ni);
      p2g_run1<M>(n, w.x, w.y, g, hk, ihk);
    }
}

// The tent mode and scale for window half-width l (tent width l == 4 ? 4h
// : h): mode 2 (positions and node coordinates scaled by inv_h) takes the
// scaled offset itself for l = 1 and a quarter of it for l = 4 (exact);
// mode 1 multiplies by inv_h (/ 4); mode 0 divides by h (4h: exact in float).
template <bool PAIR>
__device__ __forceinline__ void p2g_chunk(P2gNode& n0, P2gNode& n1, bool on1, int l, int mode, int i, int j, int k,
                                          int ni, int nj, int nk, const P2gStage& g, float h, float inv_h) {
  const bool w4 = l == 4;
  if (mode == 2 && !w4) {
    if (PAIR) p2g_chunk2<2>(n0, n1, on1, l, i, j, k, ni, nj, nk, g, h, inv_h);
    else p2g_chunk1<2>(n0, l, i, j, k, ni, nj, nk, g, h, inv_h);
  } else if (mode != 0) {
    const float ihk = mode == 2 ? 0.25f : (w4 ? inv_h * 0.25f : inv_h);
    if (PAIR) p2g_chunk2<1>(n0, n1, on1, l, i, j, k, ni, nj, nk, g, h, ihk);
    else p2g_chunk1<1>(n0, l, i, j, k, ni, nj, nk, g, h, ihk);
  } else {
    const float hk = w4 ? (float)(4.0 * (double)h) : h;
    if (PAIR) p2g_chunk2<0>(n0, n1, on1, l, i, j, k, ni, nj, nk, g, hk, inv_h);
    else p2g_chunk1<0>(n0, l, i, j, k, ni, nj, nk, g, hk, inv_h);
  }
}

template <int TZ, bool SUB>
__global__ void __launch_bounds__(P2gTile<TZ, SUB>::threads, P2gTile<TZ, SUB>::ctas_per_sm)
    p2g3_tile_kernel(const int* __restrict__ start, const float4* __restrict__ spos,
                     const float4* __restrict__ svel, float* __restrict__ fu, float* __restrict__ cu,
                     float* __restrict__ fv, float* __restrict__ cv, float* __restrict__ fw, float* __restrict__ cw,
                     int ni, int nj, int nk, float h, float inv_h, int ntx, int nty, int cap) {
  using T = P2gTile<TZ, SUB>;
  constexpr int R = T::rows_pad / 32;  // rows per lane of the scan
  constexpr int S = T::rx + 1;         // the bucket table's row stride
  extern __shared__ __align__(16) int psm[];
  int* cs = psm;                       // [row][c]: staged index of bucket clo + c's first particle
  int* rbeg = cs + T::rows * S;        // [row]: sorted index of the row run's first particle
  int* roff = rbeg + T::rows_pad;      // [row]: staged index of the row run's first particle
  const int A = p2g_slot(cap - 1) + 1;
  float* px = reinterpret_cast<float*>(psm + T::fixed_ints);
  float *py = px + A, *pz = py + A, *vx = pz + A, *vy = vx + A, *vz = vy + A;
  const int tid = threadIdx.x, t = blockIdx.x;
  const int i0 = (t % ntx) * kP2gTX, j0 = ((t / ntx) % nty) * kP2gTY, k0 = (t / (ntx * nty)) * TZ;
  // the widest window of the tile's nodes: 4 where one lies within 4 of a
  // subdomain's boundary (some axis of the tile comes that close)
  int L = 1;
  if (SUB) {
    auto near = [](int a0, int n, int w) { return a0 <= 4 || min(a0 + w - 1, n) >= n - 4; };
    if (near(i0, ni, kP2gTX) || near(j0, nj, kP2gTY) || near(k0, nk, TZ)) L = 4;
  }
  // the staged cells: [clo, chi] x [cjlo, cjhi] x [cklo, ckhi]
  const int clo = max(i0 - L, 0), chi = min(i0 + kP2gTX - 1 + L, ni - 1), nrx = chi - clo + 1;
  const int cjlo = max(j0 - L, 0), nry = min(j0 + kP2gTY - 1 + L, nj - 1) - cjlo + 1;
  const int cklo = max(k0 - L, 0), nrz = min(k0 + TZ - 1 + L, nk - 1) - cklo + 1;
  const int nrows = nry * nrz;
  auto row_base = [&](int r) { return ((cklo + r / nry) * nj + cjlo + r % nry) * ni; };
  // the region's bucket starts in one round of loads, then each row's run
  for (int e = tid; e < nrows * (nrx + 1); e += T::threads) {
    const int r = e / (nrx + 1), c = e - r * (nrx + 1);
    cs[r * S + c] = __ldg(start + row_base(r) + clo + c);
  }
  __syncthreads();
  for (int r = tid; r < T::rows_pad; r += T::threads) {
    int len = 0;
    if (r < nrows) {
      const int b = cs[r * S];
      rbeg[r] = b;
      len = cs[r * S + nrx] - b;
    }
    roff[r] = len;
  }
  __syncthreads();
  if (tid < 32) {  // exclusive scan of the run lengths, R rows per lane
    int v[R], x = 0;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      v[q] = roff[R * tid + q];
      x += v[q];
    }
    const int own = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (tid >= o) x += y;
    }
    int pre = x - own;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      roff[R * tid + q] = pre;
      pre += v[q];
    }
  }
  __syncthreads();
  for (int e = tid; e < nrows * (nrx + 1); e += T::threads) {
    const int r = e / (nrx + 1), c = e - r * (nrx + 1);
    cs[r * S + c] += roff[r] - rbeg[r];
  }
  const int total = roff[nrows];  // the rows past nrows have length 0
  // tent mode (p2g_tent): 2 scales positions and node coordinates by inv_h
  const int mode = inv_h == 0.0f ? 0 : (inv_h >= 1.0f ? 2 : 1);
  const float sc = mode == 2 ? inv_h : 1.0f;
  // copy staged indices [c0, c1) into the six arrays (positions scaled by
  // sc): each warp copies whole rows, kP2gBatch steps of 32 particles with
  // their loads in flight before the stores
  auto stage = [&](int c0, int c1, float* qx, float* qy, float* qz, float* wx, float* wy, float* wz) {
    for (int r = tid >> 5; r < nrows; r += T::threads / 32) {
      const int lo = max(roff[r], c0), hi = min(roff[r + 1], c1);
      const int g = rbeg[r] - roff[r];
      for (int s0 = lo + (tid & 31); s0 < hi; s0 += 32 * kP2gBatch) {
        float4 a[kP2gBatch], v[kP2gBatch];
#pragma unroll
        for (int q = 0; q < kP2gBatch; ++q) {
          const int s = s0 + 32 * q;
          if (s < hi) {
            a[q] = __ldg(spos + g + s);
            v[q] = __ldg(svel + g + s);
          }
        }
#pragma unroll
        for (int q = 0; q < kP2gBatch; ++q) {
          const int s = s0 + 32 * q;
          if (s < hi) {
            const int P = p2g_slot(s - c0);
            qx[P] = a[q].x * sc;
            qy[P] = a[q].y * sc;
            qz[P] = a[q].z * sc;
            wx[P] = v[q].x;
            wy[P] = v[q].y;
            wz[P] = v[q].z;
          }
        }
      }
    }
  };
  auto scale = [&](P2gNode& n) {
    n.xi *= sc;
    n.xh *= sc;
    n.yj *= sc;
    n.yh *= sc;
    n.zk *= sc;
    n.zh *= sc;
  };
  // window half-widths: SubDomainSolver::determineDist, 4 within 4 cells of the boundary
  auto half = [&](int ii, int jj, int kk) {
    if (!SUB) return 1;
    const int d = min(min(min(ii, ni - ii), min(jj, nj - jj)), min(kk, nk - kk));
    return d <= 4 ? 4 : 1;
  };
  const bool hu = fu != nullptr, hv = fv != nullptr, hw = fw != nullptr;
  const int i = i0 + tid % kP2gTX, j = j0 + (tid / kP2gTX) % kP2gTY, k = k0 + 2 * (tid / (kP2gTX * kP2gTY));
  const bool on0 = i <= ni && j <= nj && k <= nk, on1 = on0 && k + 1 <= nk;
  const int l0 = half(i, j, k), l1 = half(i, j, k + 1);
  P2gNode n0 = p2g_node(i, j, k, ni, nj, nk, h, hu, hv, hw);
  P2gNode n1 = p2g_node(i, j, k + 1, ni, nj, nk, h, hu, hv, hw);
  if (mode == 2) {
    scale(n0);
    scale(n1);
  }
  // the staged sequence is the row runs in row order (k, then j), and a
  // node's window is a sub-run of each of its rows, taken in that order:
  // chunk by chunk, each node adds the part of its window the chunk holds
  for (int c0 = 0; c0 < total; c0 += cap) {
    const int c1 = min(c0 + cap, total);
    __syncthreads();  // the previous chunk is consumed (and cs is written)
    stage(c0, c1, px, py, pz, vx, vy, vz);
    __syncthreads();
    if (!on0) continue;
    const P2gStage g{cs, S, clo, cjlo, cklo, nry, c0, c1, px, py, pz, vx, vy, vz};
    if (l0 == l1 || !on1) {
      p2g_chunk<true>(n0, n1, on1 && l0 == l1, l0, mode, i, j, k, ni, nj, nk, g, h, inv_h);
    } else {  // a subdomain node pair across the shell's edge: each alone
      p2g_chunk<false>(n0, n0, false, l0, mode, i, j, k, ni, nj, nk, g, h, inv_h);
      p2g_chunk<false>(n1, n1, false, l1, mode, i, j, k + 1, ni, nj, nk, g, h, inv_h);
    }
  }
  if (on0) p2g_store(n0, i, j, k, ni, nj, fu, cu, fv, cv, fw, cw);
  if (on1) p2g_store(n1, i, j, k + 1, ni, nj, fu, cu, fv, cv, fw, cw);
}

// particle_from_grid, Smoke_solver3D.cpp:1398-1406 (flip_ratio == 1:
// vel += trilinear(delta)); otherwise the FLIP/PIC blend of
// fluid_particle::interpolate, fluid_particle.h:315-328, evaluated in double:
// vel = (1 - f) u_new(pos) + f (vel + delta(pos)).
// Samples are taken at pos - bmin (SubDomainSolver::particle_from_grid,
// sub_domain.cpp:1161-1178, for a subdomain; origin 0 for the main grid).
__global__ void g2p_kernel(ParticleRec* __restrict__ p, int np, GridView du, GridView dv, GridView dw, GridView un,
                           GridView vn, GridView wn, double flip_ratio, SubFrame sf) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
    ParticleRec r = p[q];
    double x = r.pos[0] - sf.bx, y = r.pos[1] - sf.by, z = r.pos[2] - sf.bz;
    float d0 = sample_linear(du, x, y, z), d1 = sample_linear(dv, x, y, z), d2 = sample_linear(dw, x, y, z);
    if (flip_ratio == 1.0) {
      r.vel[0] = r.vel[0] + d0;
      r.vel[1] = r.vel[1] + d1;
      r.vel[2] = r.vel[2] + d2;
    } else {
      const double pic = 1.0 - flip_ratio;
      float s0 = sample_linear(un, x, y, z), s1 = sample_linear(vn, x, y, z), s2 = sample_linear(wn, x, y, z);
      r.vel[0] = (float)(pic * (double)s0 + flip_ratio * (double)(r.vel[0] + d0));
      r.vel[1] = (float)(pic * (double)s1 + flip_ratio * (double)(r.vel[1] + d1));
      r.vel[2] = (float)(pic * (double)s2 + flip_ratio * (double)(r.vel[2] + d2));
    }
    p[q].vel[0] = r.vel[0];
    p[q].vel[1] = r.vel[1];
    p[q].vel[2] = r.vel[2];
  }
}

// ---------------------------------------------------------------------------
// FLIP particle advection and reseeding (the steps either side of P2G/G2P)

// SmokeSolver3D::traceRK3, Smoke_solver3D.cpp:144-158, through get_velocity
// (subdomain blend inactive): c1 = 2/9 dt and c2 = 3/9 dt rounded from
// double, and c3 = (1 - c1 - c2) dt as the reference writes it (c1, c2
// already carry dt).
// `vel(x, v)` writes the velocity at x into v.
template <class F>
__device__ __forceinline__ void trace_rk3_f(F vel, const float p[3], float dt, float out[3]) {
  const float c1 = (float)(2.0 / 9.0 * (double)dt), c2 = (float)(3.0 / 9.0 * (double)dt);
  const float c3 = (float)((1.0 - (double)c1 - (double)c2) * (double)dt);
  const float half = (float)(0.5 * (double)dt), q3 = (float)(0.75 * (double)dt);
  float v1[3], v2[3], v3[3];
  vel(p, v1);
  const float m1[3] = {p[0] + half * v1[0], p[1] + half * v1[1], p[2] + half * v1[2]};
  vel(m1, v2);
  const float m2[3] = {p[0] + q3 * v2[0], p[1] + q3 * v2[1], p[2] + q3 * v2[2]};
  vel(m2, v3);
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = p[a] + c1 * v1[a] + c2 * v2[a] + c3 * v3[a];
}

__device__ __forceinline__ void trace_rk3(const GridView& u, const GridView& v, const GridView& w, const float p[3],
                                          float dt, float out[3]) {
  trace_rk3_f(
      [&](const float* x, float* o) {
        o[0] = sample_linear(u, x[0], x[1], x[2]);
        o[1] = sample_linear(v, x[0], x[1], x[2]);
        o[2] = sample_linear(w, x[0], x[1], x[2]);
      },
      p, dt, out);
}

// get_solid_normal (Smoke_solver3D.cpp:115-124): Buffer3D::sample_grad
// (fluid_buffer3D.h:249-257, differences over +-h in double world
// coordinates) normalised by mag = sqrt(mag2) + 1e-6 (vec.h:194-219; the
// square root in double, as the reference's build evaluates it)
__device__ __forceinline__ void solid_normal(const GridView& phi, const float p[3], float n[3]) {
  const double x = p[0], y = p[1], z = p[2], h = phi.h;
  const float r = sample_linear(phi, x + h, y, z), l = sample_linear(phi, x - h, y, z);
  const float u = sample_linear(phi, x, y + h, z), b = sample_linear(phi, x, y - h, z);
  const float f = sample_linear(phi, x, y, z - h), k = sample_linear(phi, x, y, z + h);
  n[0] = 0.5f * (float)((double)(r - l) / h);
  n[1] = 0.5f * (float)((double)(u - b) / h);
  n[2] = 0.5f * (float)((double)(k - f) / h);
  float m2 = n[0] * n[0];
  m2 = m2 + n[1] * n[1];
  m2 = m2 + n[2] * n[2];
  const float mag = (float)(sqrt((double)m2) + 1e-6);
  n[0] = n[0] / mag;
  n[1] = n[1] / mag;
  n[2] = n[2] / mag;
}

// The nested subdomain as the main grid's samplers see it: SmokeSolver3D's
// get_velocity, get_solid_phi and get_solid_normal (Smoke_solver3D.cpp:71-124)
// defer to SubDomainSolver (sub_domain.cpp:61-105) inside its box.
struct Nest {
  float bmin[3], bmax[3], h;
  GridView u, v, w, phi;  // the subdomain's face velocities and nodal phi (origin bmin)
};

// is_in (m = 2) and is_in2 (m = 5), sub_domain.h:176-201: strictly inside
// [bmin + m h, bmax - m h] on every axis, compared in double.
__device__ __forceinline__ bool nest_inside(const Nest& n, const float p[3], double m) {
  bool in = true;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    in = in && (double)p[a] > (double)n.bmin[a] + m * (double)n.h &&
         (double)p[a] < (double)n.bmax[a] - m * (double)n.h;
  return in;
}

// get_boundary_coef, sub_domain.cpp:96-105: the smallest |component| of the
// offsets to the corners of the box 5h inside the subdomain, over 4h,
// clamped to [0, 1]; float throughout.
__device__ __forceinline__ float nest_coef(const Nest& n, const float p[3]) {
  const float m5 = 5.0f * n.h;
  float d1 = fabsf(p[0] - (n.bmin[0] + m5)), d2 = fabsf(p[0] - (n.bmax[0] - m5));
#pragma unroll
  for (int a = 1; a < 3; ++a) {
    const float e1 = fabsf(p[a] - (n.bmin[a] + m5)), e2 = fabsf(p[a] - (n.bmax[a] - m5));
    if (e1 < d1) d1 = e1;
    if (e2 < d2) d2 = e2;
  }
  const float c = __fdiv_rn(d2 < d1 ? d2 : d1, 4.0f * n.h);
  return c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
}

// get_velocity: the main grid's sample, replaced inside is_in2 by
// c v_sub + (1 - c) v with v_sub sampled at pos - bmin.
__device__ __forceinline__ void nested_velocity(const GridView& u, const GridView& v, const GridView& w,
                                                const Nest& n, const float p[3], float o[3]) {
  o[0] = sample_linear(u, p[0], p[1], p[2]);
  o[1] = sample_linear(v, p[0], p[1], p[2]);
  o[2] = sample_linear(w, p[0], p[1], p[2]);
  if (nest_inside(n, p, 5.0)) {
    const float q0 = p[0] - n.bmin[0], q1 = p[1] - n.bmin[1], q2 = p[2] - n.bmin[2];
    const float s[3] = {sample_linear(n.u, q0, q1, q2), sample_linear(n.v, q0, q1, q2),
                        sample_linear(n.w, q0, q1, q2)};
    const float c = nest_coef(n, p), c1 = 1.0f - c;
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = __fadd_rn(__fmul_rn(c, s[a]), __fmul_rn(c1, o[a]));
  }
}

// get_solid_phi: the subdomain's nodal phi at pos - bmin inside is_in.
__device__ __forceinline__ float nested_phi(const GridView& phi, const Nest& n, const float p[3]) {
  if (nest_inside(n, p, 2.0)) return sample_linear(n.phi, p[0] - n.bmin[0], p[1] - n.bmin[1], p[2] - n.bmin[2]);
  return sample_linear(phi, p[0], p[1], p[2]);
}

// get_solid_normal: the subdomain's phi gradient (its own h) inside is_in,
// normalised like the main grid's.
__device__ __forceinline__ void nested_normal(const GridView& phi, const Nest& n, const float p[3], float o[3]) {
  if (nest_inside(n, p, 2.0)) {
    const float q[3] = {p[0] - n.bmin[0], p[1] - n.bmin[1], p[2] - n.bmin[2]};
    solid_normal(n.phi, q, o);
  } else {
    solid_normal(phi, p, o);
  }
}

// SmokeSolver3D::advect_FLIP, Smoke_solver3D.cpp:1407-1449: RK3 through the
// grid velocity, then out of a solid along its normal by -phi.  NEST: the
// velocity, phi and normal of the main grid with its subdomain active.
template <bool NEST>
__global__ void advect_flip_kernel(ParticleRec* __restrict__ p, int np, GridView u, GridView v, GridView w,
                                   GridView phi, float dt, Nest nest) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
    const float pos0[3] = {p[q].pos[0], p[q].pos[1], p[q].pos[2]};
    float pos[3];
    if (NEST)
      trace_rk3_f([&](const float* x, float* o) { nested_velocity(u, v, w, nest, x, o); }, pos0, dt, pos);
    else
      trace_rk3(u, v, w, pos0, dt, pos);
    const float ph = NEST ? nested_phi(phi, nest, pos) : sample_linear(phi, pos[0], pos[1], pos[2]);
    if (ph < 0) {
      float n[3];
      if (NEST)
        nested_normal(phi, nest, pos, n);
      else
        solid_normal(phi, pos, n);
#pragma unroll
      for (int a = 0; a < 3; ++a) pos[a] = pos[a] - ph * n[a];
    }
    p[q].pos[0] = pos[0];
    p[q].pos[1] = pos[1];
    p[q].pos[2] = pos[2];
  }
}

// Counter-based uniform in [-1, 1) for reseeding: a 32-bit integer mix of
// (seed, cell, slot, axis).  The reference draws frand(-1, 1) from rand()
// (Smoke_solver3D.h:36-39) - the same distribution from a sequential
// generator that parallel code cannot reproduce.
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float reseed_uniform(uint32_t seed, uint32_t cell, uint32_t slot, uint32_t axis) {
  const uint32_t r = mix32(mix32(mix32(seed ^ 0x9e3779b9u) + cell) + (slot * 3u + axis));
  return -1.0f + 2.0f * ((float)(r >> 8) * (1.0f / 16777216.0f));
}

// reorder_FLIP, Smoke_solver3D.cpp:1347-1396: particles written per cell -
// fewer than 8: all kept + topped up to 8; 8 or 9: all; 10+: the first 8
// For a subdomain (sub != 0) only the interior cells (1 .. n-2 on every
// axis) are walked (SubDomainSolver::reorder_FLIP, sub_domain.cpp:1110-1159).
__device__ __forceinline__ bool reorder_cell(int c, int ni, int nj, int nk, int sub) {
  if (!sub) return true;
  const int i = c % ni, j = (c / ni) % nj, k = c / (ni * nj);
  return i >= 1 && i < ni - 1 && j >= 1 && j < nj - 1 && k >= 1 && k < nk - 1;
}

__global__ void reorder_count_kernel(const int* __restrict__ start, int* __restrict__ out_count, int nc, int ni,
                                     int nj, int nk, int sub) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const int cnt = start[c + 1] - start[c];
    out_count[c] = !reorder_cell(c, ni, nj, nk, sub) ? 0 : (cnt < 8 ? 8 : (cnt < 10 ? cnt : 8));
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out_count[nc] = 0;
}

// one thread per cell: kept particles in bucket order, then the new ones at
// bmin + (i, j, k) h + r 0.49 h with the grid velocity there (sampled at
// pos - bmin), density and temperature 0 (get_velocity_self,
// Smoke_solver3D.cpp:89-97; SubDomainSolver::get_velocity, sub_domain.cpp:69-76)
__global__ void reorder_write_kernel(const ParticleRec* __restrict__ p, const int* __restrict__ start,
                                     const int* __restrict__ order, const int* __restrict__ base,
                                     ParticleRec* __restrict__ tmp, int ni, int nj, int nk, float h, GridView u,
                                     GridView v, GridView w, uint32_t seed, SubFrame sf) {
  const int nc = ni * nj * nk;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    if (!reorder_cell(c, ni, nj, nk, sf.sub)) continue;
    const int s0 = start[c], cnt = start[c + 1] - s0, b = base[c];
    const int keep = cnt < 10 ? cnt : 8;
    for (int e = 0; e < keep; ++e) tmp[b + e] = p[order[s0 + e]];
    if (cnt < 8) {
      const int i = c % ni, j = (c / ni) % nj, k = c / (ni * nj);
      const float bx = sf.bx + (float)i * h, by = sf.by + (float)j * h, bz = sf.bz + (float)k * h;
      for (int e = cnt; e < 8; ++e) {
        ParticleRec r;
        r.pos[0] = bx + reseed_uniform(seed, (uint32_t)c, (uint32_t)e, 0u) * 0.49f * h;
        r.pos[1] = by + reseed_uniform(seed, (uint32_t)c, (uint32_t)e, 1u) * 0.49f * h;
        r.pos[2] = bz + reseed_uniform(seed, (uint32_t)c, (uint32_t)e, 2u) * 0.49f * h;
        const float q0 = r.pos[0] - sf.bx, q1 = r.pos[1] - sf.by, q2 = r.pos[2] - sf.bz;
        r.vel[0] = sample_linear(u, q0, q1, q2);
        r.vel[1] = sample_linear(v, q0, q1, q2);
        r.vel[2] = sample_linear(w, q0, q1, q2);
        r.dens = 0.0f;
        r.temp = 0.0f;
        r.hash_idx = 0;
        r.sub_hash_idx = 0;
        tmp[b + e] = r;
      }
    }
  }
}

// keep flag: sampled solid phi >= 0 (reorder_FLIP's final filter); with
// `nested` the main grid's get_solid_phi with its subdomain active.
__global__ void solid_keep_kernel(const ParticleRec* __restrict__ tmp, const int* __restrict__ total,
                                  int* __restrict__ keep, GridView phi, int cap, SubFrame sf, int nested, Nest nest) {
  const int n = min(*total, cap);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float x[3] = {tmp[q].pos[0] - sf.bx, tmp[q].pos[1] - sf.by, tmp[q].pos[2] - sf.bz};
    keep[q] = (nested ? nested_phi(phi, nest, x) : sample_linear(phi, x[0], x[1], x[2])) >= 0.0f ? 1 : 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) keep[n] = 0;
}

// The halo selection of SmokeSolver3D::time_step (Smoke_solver3D.cpp:390-398):
// flag the particles strictly inside [bmin - dx, bmax + dx] on every axis
// (SubDomainSolver::is_halo, sub_domain.h:202-213; float).
__global__ void halo_flag_kernel(const ParticleRec* __restrict__ p, int np, Nest nest, float dx,
                                 int* __restrict__ flag) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= np; q += gridDim.x * blockDim.x) {
    int f = 0;
    if (q < np) {
      f = 1;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float x = p[q].pos[a];
        f &= (x > nest.bmin[a] - dx && x < nest.bmax[a] + dx) ? 1 : 0;
      }
    }
    flag[q] = f;
  }
}

__global__ void halo_compact_kernel(const ParticleRec* __restrict__ p, int np, const int* __restrict__ flag,
                                    const int* __restrict__ pos, ParticleRec* __restrict__ out, int cap) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x)
    if (flag[q] && pos[q] < cap) out[pos[q]] = p[q];
}

__global__ void compact_kernel(const ParticleRec* __restrict__ tmp, const int* __restrict__ keep,
                               const int* __restrict__ pos, const int* __restrict__ total, ParticleRec* __restrict__ out,
                               int cap_in, int cap_out) {
  const int n = min(*total, cap_in);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    if (keep[q] && pos[q] < cap_out) out[pos[q]] = tmp[q];
}

}  // namespace vflip
