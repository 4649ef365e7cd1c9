// The grid advection forms of SmokeSolver3D beside the RK2-linear one, and
// the smoke scalars on the doubled density/temperature grids:
//
//   advect_field_cubic_clamp (Smoke_solver3D.cpp:657-707): the RK2 midpoint
//     backtrace, a cubic sample of the 4x4x4 neighbourhood, replaced by the
//     trilinear sample where it reaches or leaves the range of the eight
//     surrounding nodes.  SmokeSolver3D::advect (:8-29) applies it to u, v, w.
//   advect_field (:564-610): traceRK3 with step -dt, trilinear sample; used
//     for density and temperature, which live on 2ni x 2nj x 2nk grids at
//     h/2 (Smoke_solver3D.h:313-315).
//   gen_heat (:1624-1650) and add_smokeforce (:1652-1668).
//
// EXACT instantiations keep the reference's FP64 world->grid transform,
// FP64 lerps and FP64 cubic sums with float weights, so they are bit-identical
// to it (the library is built with -fmad=false); the others run the same
// scheme in FP32 with fused multiply-adds.
#pragma once
#include <type_traits>

#include "transfer_kernels.cuh"

namespace vflip {

// Buffer3D::cubic_interp_weights (fluid_buffer3D.h:22-29) with T = float.
__device__ __forceinline__ void cubic_weights(float f, float w[4]) {
  const float f2 = f * f, f3 = f2 * f;
  w[0] = -(float)(1. / 3) * f + 0.5f * f2 - (float)(1. / 6) * f3;
  w[1] = 1.0f - f2 + 0.5f * (f3 - f);
  w[2] = f + 0.5f * (f2 - f3);
  w[3] = (float)(1. / 6) * (f3 - f);
}

// Buffer3D::cubic_interp (fluid_buffer3D.h:31-38): the weighted sum, left to
// right; in double (float weights widened) for EXACT.
template <bool EXACT, typename R>
__device__ __forceinline__ R cubic_sum(const float w[4], R a, R b, R c, R d) {
  if constexpr (EXACT) {
    return (double)w[0] * a + (double)w[1] * b + (double)w[2] * c + (double)w[3] * d;
  } else {
    return __fmaf_rn(w[3], d, __fmaf_rn(w[2], c, __fmaf_rn(w[1], b, w[0] * a)));
  }
}

// Buffer3D::sample_cubic (fluid_buffer3D.h:259-326) with the clamp of
// advect_field_cubic_clamp (Smoke_solver3D.cpp:693-703).  The 64 clamped
// nodes are read row by row (z outer, y inner, as the reference sums them);
// the eight nodes around the point are the middle of that block, so the
// trilinear fallback (sample_cube_lerp, fluid_buffer3D.h:329-356) and the
// corner range reuse them.
template <bool EXACT>
__device__ __forceinline__ float sample_cubic_clamp(const GridView& g, float px, float py, float pz) {
  using R = typename std::conditional<EXACT, double, float>::type;
  R gx, gy, gz;
  if constexpr (EXACT) {
    gx = div_h(px, g) + g.ox;
    gy = div_h(py, g) + g.oy;
    gz = div_h(pz, g) + g.oz;
  } else {
    const float ih = (float)(g.inv_h != 0.0 ? g.inv_h : 1.0 / g.h);
    gx = __fmaf_rn(px, ih, (float)g.ox);
    gy = __fmaf_rn(py, ih, (float)g.oy);
    gz = __fmaf_rn(pz, ih, (float)g.oz);
  }
  const int i = (int)floor(gx), j = (int)floor(gy), k = (int)floor(gz);
  const R x = gx - (R)i, y = gy - (R)j, z = gz - (R)k;
  float wx[4], wy[4], wz[4];
  cubic_weights((float)x, wx);
  cubic_weights((float)y, wy);
  cubic_weights((float)z, wz);
  const int sy = g.nx, sz = g.nx * g.ny;
  int I[4], J[4], K[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    I[t] = clampi(i - 1 + t, g.nx - 1);
    J[t] = clampi(j - 1 + t, g.ny - 1) * sy;
    K[t] = clampi(k - 1 + t, g.nz - 1) * sz;
  }
  float cn[8];  // node (i+di, j+dj, k+dk) at cn[di + 2 dj + 4 dk]
  R fz[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    R fy[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const float* row = g.d + (J[b] + K[c]);
      const float a0 = __ldg(row + I[0]), a1 = __ldg(row + I[1]), a2 = __ldg(row + I[2]), a3 = __ldg(row + I[3]);
      fy[b] = cubic_sum<EXACT, R>(wx, (R)a0, (R)a1, (R)a2, (R)a3);
      if ((b == 1 || b == 2) && (c == 1 || c == 2)) {
        cn[2 * (b - 1) + 4 * (c - 1)] = a1;
        cn[1 + 2 * (b - 1) + 4 * (c - 1)] = a2;
      }
    }
    fz[c] = cubic_sum<EXACT, R>(wy, fy[0], fy[1], fy[2], fy[3]);
  }
  const float cubic = (float)cubic_sum<EXACT, R>(wz, fz[0], fz[1], fz[2], fz[3]);
  float lo = cn[0], hi = cn[0];
#pragma unroll
  for (int t = 1; t < 8; ++t) {
    lo = fminf(lo, cn[t]);
    hi = fmaxf(hi, cn[t]);
  }
  if (!(cubic <= lo || cubic >= hi)) return cubic;
  if constexpr (EXACT) {
    const double v1 = lerp_d(lerp_d(cn[0], cn[1], x), lerp_d(cn[2], cn[3], x), y);
    const double v2 = lerp_d(lerp_d(cn[4], cn[5], x), lerp_d(cn[6], cn[7], x), y);
    return (float)lerp_d(v1, v2, z);
  } else {
    const float v1 = lerp_f(lerp_f(cn[0], cn[1], x), lerp_f(cn[2], cn[3], x), y);
    const float v2 = lerp_f(lerp_f(cn[4], cn[5], x), lerp_f(cn[6], cn[7], x), y);
    return lerp_f(v1, v2, z);
  }
}

// The RK2 midpoint backtrace of SubDomainSolver::advect_field
// (sub_domain.cpp:210-222) and advect_field_cubic_clamp
// (Smoke_solver3D.cpp:682-691): the half step in double, the full step in
// float (EXACT), or both in float.
template <bool EXACT>
__device__ __forceinline__ void rk2_backtrace(const GridView& u, const GridView& v, const GridView& w, float dt,
                                              float wx, float wy, float wz, float p[3]) {
  float a = smp<EXACT>(u, wx, wy, wz), b = smp<EXACT>(v, wx, wy, wz), c = smp<EXACT>(w, wx, wy, wz);
  float px, py, pz;
  if constexpr (EXACT) {
    const double hdt = 0.5 * (double)dt;
    px = (float)((double)wx - hdt * (double)a);
    py = (float)((double)wy - hdt * (double)b);
    pz = (float)((double)wz - hdt * (double)c);
  } else {
    const float hf = 0.5f * dt;
    px = wx - hf * a;
    py = wy - hf * b;
    pz = wz - hf * c;
  }
  a = smp<EXACT>(u, px, py, pz);
  b = smp<EXACT>(v, px, py, pz);
  c = smp<EXACT>(w, px, py, pz);
  p[0] = wx - dt * a;
  p[1] = wy - dt * b;
  p[2] = wz - dt * c;
}

// Node (i,j,k) of a grid at world ((i-ox)h, (j-oy)h, (k-oz)h), rounded to
// float from double as `((float)i - field._ox) * _hx` is.
__device__ __forceinline__ void node_world_d(const GridView& f, unsigned e, double h, float p[3]) {
  const unsigned row = e / (unsigned)f.nx;
  const int i = (int)(e - row * (unsigned)f.nx), j = (int)(row % (unsigned)f.ny), k = (int)(row / (unsigned)f.ny);
  p[0] = (float)(((double)(float)i - f.ox) * h);
  p[1] = (float)(((double)(float)j - f.oy) * h);
  p[2] = (float)(((double)(float)k - f.oz) * h);
}

// Up to three fields (u, v, w of SmokeSolver3D::advect) in one launch:
// blockIdx.y picks the field, each block owns a contiguous run of
// `per_block` of its nodes.
struct CubicFields {
  GridView f[3];
  float* out[3];
};

template <bool EXACT>
__global__ void __launch_bounds__(256) advect_cubic_clamp_kernel(GridView u, GridView v, GridView w, CubicFields job,
                                                                 float h, float dt, int per_block) {
  const GridView& f = job.f[blockIdx.y];
  float* __restrict__ out = job.out[blockIdx.y];
  const unsigned n = (unsigned)f.nx * f.ny * f.nz;  // < 2^31, checked by the host
  const unsigned beg = blockIdx.x * (unsigned)per_block;
  if (beg >= n) return;
  const unsigned end = n - beg > (unsigned)per_block ? beg + per_block : n;
  for (unsigned e = beg + threadIdx.x; e < end; e += blockDim.x) {
    float wp[3], p[3];
    node_world_d(f, e, (double)h, wp);
    rk2_backtrace<EXACT>(u, v, w, dt, wp[0], wp[1], wp[2], p);
    out[e] = sample_cubic_clamp<EXACT>(f, p[0], p[1], p[2]);
  }
}

// SmokeSolver3D::traceRK3 (Smoke_solver3D.cpp:144-157) in FP32 for the
// non-EXACT instantiations; EXACT uses trace_rk3.
__device__ __forceinline__ void trace_rk3_f(const GridView& u, const GridView& v, const GridView& w, const float p[3],
                                            float dt, float out[3]) {
  const float c1 = (2.0f / 9.0f) * dt, c2 = (3.0f / 9.0f) * dt, c3 = (1.0f - c1 - c2) * dt;
  const float half = 0.5f * dt, q3 = 0.75f * dt;
  const float v1[3] = {sample_linear_f(u, p[0], p[1], p[2]), sample_linear_f(v, p[0], p[1], p[2]),
                       sample_linear_f(w, p[0], p[1], p[2])};
  const float m1[3] = {__fmaf_rn(half, v1[0], p[0]), __fmaf_rn(half, v1[1], p[1]), __fmaf_rn(half, v1[2], p[2])};
  const float v2[3] = {sample_linear_f(u, m1[0], m1[1], m1[2]), sample_linear_f(v, m1[0], m1[1], m1[2]),
                       sample_linear_f(w, m1[0], m1[1], m1[2])};
  const float m2[3] = {__fmaf_rn(q3, v2[0], p[0]), __fmaf_rn(q3, v2[1], p[1]), __fmaf_rn(q3, v2[2], p[2])};
  const float v3[3] = {sample_linear_f(u, m2[0], m2[1], m2[2]), sample_linear_f(v, m2[0], m2[1], m2[2]),
                       sample_linear_f(w, m2[0], m2[1], m2[2])};
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = __fmaf_rn(c3, v3[a], __fmaf_rn(c2, v2[a], __fmaf_rn(c1, v1[a], p[a])));
}

// SmokeSolver3D::advect_field (Smoke_solver3D.cpp:564-610) for one or two
// fields on the same grid (density and temperature share the backtrace).
template <bool EXACT>
__global__ void __launch_bounds__(256) advect_rk3_kernel(GridView u, GridView v, GridView w, GridView f,
                                                         float* __restrict__ out, GridView f2,
                                                         float* __restrict__ out2, float dt, int per_block) {
  const unsigned n = (unsigned)f.nx * f.ny * f.nz;  // < 2^31, checked by the host
  const unsigned beg = blockIdx.x * (unsigned)per_block;
  const unsigned end = n - beg > (unsigned)per_block ? beg + per_block : n;
  for (unsigned e = beg + threadIdx.x; e < end; e += blockDim.x) {
    float p[3], b[3];
    node_world_d(f, e, f.h, p);
    if constexpr (EXACT) {
      trace_rk3(u, v, w, p, -dt, b);
    } else {
      trace_rk3_f(u, v, w, p, -dt, b);
    }
    out[e] = smp<EXACT>(f, b[0], b[1], b[2]);
    if (out2) out2[e] = smp<EXACT>(f2, b[0], b[1], b[2]);
  }
}

// SmokeSolver3D::gen_heat (Smoke_solver3D.cpp:1624-1650): decay, then the
// source cylinder (radius r about (cx, cz) in float, |y - cy| <= r/4 in
// double).  Node (i,j,k) sits at (i,j,k) * (float)fh.
struct HeatSource {
  float dt, dens_decay, temp_decay, cx, cy, cz, radius, dens, heat;
};

// 32-bit index arithmetic (the host checks nx*ny*nz < 2^31).
__global__ void gen_heat_kernel(float* __restrict__ rho, float* __restrict__ temp, int nx, int ny, int nz, float hf,
                                HeatSource s) {
  const unsigned n = (unsigned)nx * ny * nz;
  const float dr = 1.0f + s.dens_decay * s.dt, dtm = 1.0f + s.temp_decay * s.dt;
  const double band = 0.25 * (double)s.radius;
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const unsigned row = e / (unsigned)nx;
    const int i = (int)(e - row * (unsigned)nx), j = (int)(row % (unsigned)ny), k = (int)(row / (unsigned)ny);
    float r = __fdiv_rn(rho[e], dr), t = __fdiv_rn(temp[e], dtm);
    const float dx = (float)i * hf - s.cx, dz = (float)k * hf - s.cz;
    const float d = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dz, dz)));
    if (d <= s.radius && (double)fabsf((float)j * hf - s.cy) <= band) {
      r = s.dens;
      t = s.heat;
    }
    rho[e] = r;
    temp[e] = t;
  }
}

// SmokeSolver3D::add_smokeforce (Smoke_solver3D.cpp:1652-1668): y velocity
// += dt (-alpha rho + beta T), rho and T sampled trilinearly (FP64 lerps).
__global__ void add_smokeforce_kernel(ParticleRec* __restrict__ p, int np, GridView rho, GridView temp, float alpha,
                                      float beta, float dt) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
    const float x = p[q].pos[0], y = p[q].pos[1], z = p[q].pos[2];
    const float r = sample_linear(rho, x, y, z), t = sample_linear(temp, x, y, z);
    const float fy = dt * (-alpha * r + beta * t);
    p[q].vel[0] = p[q].vel[0] + 0.0f;  // the reference adds Vec3f(0, fy, 0)
    p[q].vel[1] = p[q].vel[1] + fy;
    p[q].vel[2] = p[q].vel[2] + 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Smoke tracers, SmokeSolver3D::emit_tracers / advect_tracers / write_tracers
// (Smoke_solver3D.h:46-160): float4 records (x, y, z, density).

// emit_tracers' keep test (Smoke_solver3D.h:52-59): inside [2h, L-2h] on
// every axis (float) and density > 0.01 (compared in double).
__device__ __forceinline__ bool tracer_kept(const float4 t, float h, float lx, float ly, float lz) {
  const float m = 2 * h;
  return t.x > m && t.y > m && t.z > m && t.x < lx - m && t.y < ly - m && t.z < lz - m && (double)t.w > 0.01;
}

__global__ void tracer_keep_kernel(const float4* __restrict__ tr, int n, float h, float lx, float ly, float lz,
                                   int* __restrict__ keep) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    keep[q] = tracer_kept(tr[q], h, lx, ly, lz) ? 1 : 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) keep[n] = 0;
}

__global__ void tracer_compact_kernel(const float4* __restrict__ tr, int n, const int* __restrict__ keep,
                                      const int* __restrict__ pos, float4* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    if (keep[q]) out[pos[q]] = tr[q];
}

// New tracer `slot` after the *base kept ones: the first of up to 64
// attempts whose offset, uniform in [-r, r)^3 from the counter hash of
// (seed, slot, attempt, axis), has x^2 + z^2 + y^2 <= r^2 (the reference's
// rejection test and sum order; it samples rand() over the cube of
// half-width r + h, which gives the same uniform law in the sphere).
__global__ void tracer_emit_kernel(float4* __restrict__ out, const int* __restrict__ base, int count, uint32_t seed,
                                   float r, float cx, float cy, float cz) {
  const int m = *base;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
    float ox = 0.0f, oy = 0.0f, oz = 0.0f;
    for (uint32_t a = 0; a < 64; ++a) {
      const float x = r * reseed_uniform(seed ^ 0x7f4a7c15u, (uint32_t)s, a, 0);
      const float y = r * reseed_uniform(seed ^ 0x7f4a7c15u, (uint32_t)s, a, 1);
      const float z = r * reseed_uniform(seed ^ 0x7f4a7c15u, (uint32_t)s, a, 2);
      if (x * x + z * z + y * y <= r * r) {
        ox = x;
        oy = y;
        oz = z;
        break;
      }
    }
    out[m + s] = make_float4(cx + ox, cy + oy, cz + oz, 1.0f);
  }
}

// The nested subdomain's tracer seeding of emit_tracers
// (Smoke_solver3D.h:86-96): four candidates per subdomain cell (k, j, i
// order) at bmin + (i, j, k) h + r h with r uniform in [0, 1)^3, kept where
// the main grid's get_solid_phi with the subdomain active lies in (0, h).
// The reference draws r from rand(); here it is the 24 high bits of a
// counter-based hash of (seed, cell, slot, axis).
__device__ __forceinline__ float unit_uniform(uint32_t seed, uint32_t cell, uint32_t slot, uint32_t axis) {
  const uint32_t r = mix32(mix32(mix32(seed ^ 0x2545f491u) + cell) + (slot * 3u + axis));
  return (float)(r >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ bool tracer_seed(const GridView& phi, const Nest& n, int sni, int snj, uint32_t seed, int e,
                                            float pos[3]) {
  const int c = e >> 2, slot = e & 3;
  int i, j, k;
  decode3((size_t)c, sni, snj, i, j, k);
  const float ijk[3] = {(float)i, (float)j, (float)k};
#pragma unroll
  for (int a = 0; a < 3; ++a)
    pos[a] = (n.bmin[a] + ijk[a] * n.h) + unit_uniform(seed, (uint32_t)c, (uint32_t)slot, (uint32_t)a) * n.h;
  const float ph = nested_phi(phi, n, pos);
  return ph > 0.0f && ph < n.h;
}

// flag[e] for the ncand = 4 * subdomain cells candidates; flag[ncand] = 0
__global__ void tracer_seed_flag_kernel(GridView phi, Nest n, int sni, int snj, uint32_t seed, int ncand,
                                        int* __restrict__ flag) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e <= ncand; e += gridDim.x * blockDim.x) {
    float pos[3];
    flag[e] = e < ncand && tracer_seed(phi, n, sni, snj, seed, e, pos) ? 1 : 0;
  }
}

__global__ void tracer_seed_write_kernel(GridView phi, Nest n, int sni, int snj, uint32_t seed, int ncand,
                                         const int* __restrict__ flag, const int* __restrict__ pos, int base,
                                         float4* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ncand; e += gridDim.x * blockDim.x) {
    if (!flag[e]) continue;
    float x[3];
    tracer_seed(phi, n, sni, snj, seed, e, x);
    out[base + pos[e]] = make_float4(x[0], x[1], x[2], 1.0f);
  }
}

// advect_tracers (Smoke_solver3D.h:99-120): traceRK3 with step dt, out of a
// solid along its normal where the sampled phi is <= 0, density / (1 +
// decay*dt) with the product in float and the rest in double.  NEST: the
// main grid's samplers with its subdomain active.
template <bool NEST>
__global__ void advect_tracers_kernel(float4* __restrict__ tr, int n, GridView u, GridView v, GridView w,
                                      GridView phi, float dt, float dens_decay, Nest nest) {
  const double den = 1.0 + (double)(dens_decay * dt);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float4 t = tr[q];
    const float p0[3] = {t.x, t.y, t.z};
    float pos[3];
    if (NEST)
      trace_rk3_f([&](const float* x, float* o) { nested_velocity(u, v, w, nest, x, o); }, p0, dt, pos);
    else
      trace_rk3(u, v, w, p0, dt, pos);
    const float ph = NEST ? nested_phi(phi, nest, pos) : sample_linear(phi, pos[0], pos[1], pos[2]);
    if (ph <= 0) {
      float nrm[3];
      if (NEST)
        nested_normal(phi, nest, pos, nrm);
      else
        solid_normal(phi, pos, nrm);
#pragma unroll
      for (int a = 0; a < 3; ++a) pos[a] = pos[a] - ph * nrm[a];
    }
    tr[q] = make_float4(pos[0], pos[1], pos[2], (float)((double)t.w / den));
  }
}

// write_tracers' records (Smoke_solver3D.h:128-140): (x/lx - 0.5, y/lx,
// z/lx - 0.5, density), the subtraction in double.
__global__ void tracer_records_kernel(const float4* __restrict__ tr, int n, float lx, float4* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float4 t = tr[q];
    out[q] = make_float4((float)((double)__fdiv_rn(t.x, lx) - 0.5), __fdiv_rn(t.y, lx),
                         (float)((double)__fdiv_rn(t.z, lx) - 0.5), t.w);
  }
}

}  // namespace vflip
