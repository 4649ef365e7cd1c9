// Pressure-projection kernels around the solve: face weights, inflow
// overwrite, matrix-free assembly of the 7-point operator and right-hand
// side, gradient update.  Each follows SmokeSolver3D::pcg_projection
// (Smoke_Solver/Smoke_solver3D.cpp:874-1202) with the reference's float /
// double mix and order of operations, so the FP64 operator and rhs equal the
// reference's SparseMatrixd/rhs entry for entry.
#pragma once
#include "common.cuh"

namespace vflip {

// fraction_inside, levelset_util.cpp:4-13
__device__ __forceinline__ float frac2(float l, float r) {
  if (l < 0 && r < 0) return 1.0f;
  if (l < 0 && r >= 0) return l / (l - r);
  if (l >= 0 && r < 0) return r / (r - l);
  return 0.0f;
}

__device__ __forceinline__ void rot4(float& a, float& b, float& c, float& d) {
  float t = a;
  a = b; b = c; c = d; d = t;
}

// fraction_inside of a square, levelset_util.cpp:23-103.  The corner list is
// (bl, br, tr, tl) and is rotated exactly as the reference rotates it.  The
// reference's rotation loops never end when the corners that count as inside
// (phi <= 0) include exact zeros in some patterns (e.g. phi = {0, 0, 1, 1});
// here each loop is bounded by the four possible rotations and a failed
// search returns -1, after which the caller re-evaluates with exact zeros
// moved to the smallest positive float (the limit from the outside).
__device__ __forceinline__ float frac4_try(float bl, float br, float tl, float tr) {
  int inside = (bl <= 0) + (tl <= 0) + (br <= 0) + (tr <= 0);
  float q0 = bl, q1 = br, q2 = tr, q3 = tl;
  if (inside == 4) return 1.0f;
  if (inside == 3) {
    int n = 0;
    while (q0 < 0) { if (++n > 4) return -1.0f; rot4(q0, q1, q2, q3); }
    float s0 = 1 - frac2(q0, q3);
    float s1 = 1 - frac2(q0, q1);
    return 1 - 0.5f * s0 * s1;
  }
  if (inside == 2) {
    int n = 0;
    while (q0 >= 0 || !(q1 < 0 || q2 < 0)) { if (++n > 4) return -1.0f; rot4(q0, q1, q2, q3); }
    if (q1 < 0) return 0.5f * (frac2(q0, q3) + frac2(q1, q2));
    float mid = 0.25f * (q0 + q1 + q2 + q3);
    if (mid < 0) {
      float area = 0;
      float s1 = 1 - frac2(q0, q3);
      float s3 = 1 - frac2(q2, q3);
      area += 0.5f * s1 * s3;
      float s2 = 1 - frac2(q2, q1);
      float s0 = 1 - frac2(q0, q1);
      area += 0.5f * s0 * s2;
      return 1 - area;
    }
    float area = 0;
    float s0 = frac2(q0, q1);
    float s1 = frac2(q0, q3);
    area += 0.5f * s0 * s1;
    float s2 = frac2(q2, q1);
    float s3 = frac2(q2, q3);
    area += 0.5f * s2 * s3;
    return area;
  }
  if (inside == 1) {
    int n = 0;
    while (q0 >= 0) { if (++n > 4) return -1.0f; rot4(q0, q1, q2, q3); }
    float s0 = frac2(q0, q3);
    float s1 = frac2(q0, q1);
    return 0.5f * s0 * s1;
  }
  return 0.0f;
}

__device__ __forceinline__ float nudge_zero(float x) { return x == 0.0f ? 1.17549435e-38f : x; }

__device__ __forceinline__ float frac4(float bl, float br, float tl, float tr) {
  float f = frac4_try(bl, br, tl, tr);
  if (f < 0.0f) f = frac4_try(nudge_zero(bl), nudge_zero(br), nudge_zero(tl), nudge_zero(tr));
  return f;
}

__device__ __forceinline__ float clamp01(float a) { return a < 0.0f ? 0.0f : (a > 1.0f ? 1.0f : a); }

// compute_face_weights, Smoke_solver3D.cpp:874-944: weight = 1 - the
// fraction of each face inside the solid, from the nodal phi at its four
// corners (the reference's corner order per face grid).  One thread per node
// (i, j, k) of the (ni+1) x (nj+1) x (nk+1) lattice writes the u, v and w
// faces whose lower corner that node is, so seven nodal phi loads serve the
// three faces, and the 2-D block over (i, j) with z over the grid needs no
// index division.
__global__ void face_weights3_kernel(const float* __restrict__ phi, float* __restrict__ uw, float* __restrict__ vw,
                                     float* __restrict__ ww, int ni, int nj, int nk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
  if (i > ni || j > nj || k > nk) return;
  const int px = ni + 1, py = nj + 1;
  auto P = [&](int a, int b, int c) { return __ldg(phi + lin3(a, b, c, px, py)); };
  const bool xi = i < ni, yj = j < nj, zk = k < nk;
  // all seven corners loaded up front (one round of memory latency)
  const float p000 = P(i, j, k);
  const float p010 = yj ? P(i, j + 1, k) : 0.0f;
  const float p001 = zk ? P(i, j, k + 1) : 0.0f;
  const float p100 = xi ? P(i + 1, j, k) : 0.0f;
  const float p011 = (yj && zk) ? P(i, j + 1, k + 1) : 0.0f;
  const float p101 = (xi && zk) ? P(i + 1, j, k + 1) : 0.0f;
  const float p110 = (xi && yj) ? P(i + 1, j + 1, k) : 0.0f;
  if (yj && zk) uw[lin3(i, j, k, ni + 1, nj)] = clamp01(1 - frac4(p000, p010, p001, p011));
  if (xi && zk) vw[lin3(i, j, k, ni, nj + 1)] = clamp01(1 - frac4(p000, p001, p100, p101));
  if (xi && yj) ww[lin3(i, j, k, ni, nj)] = clamp01(1 - frac4(p000, p010, p100, p110));
}

// Inflow overwrite, Smoke_solver3D.cpp:964-980: every cell with b_desc == 1
// pins its six faces (u = U_in, v = w = 0).  Concurrent writers store the
// same value, so the result is order independent.
__global__ void inflow_kernel(const int8_t* __restrict__ bdesc, float* __restrict__ u, float* __restrict__ v,
                              float* __restrict__ w, float U_in, int ni, int nj, int nk) {
  const size_t n = (size_t)ni * nj * nk;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    if (bdesc[e] != 1) continue;
    int i, j, k;
    decode3(e, ni, nj, i, j, k);
    u[lin3(i, j, k, ni + 1, nj)] = U_in;
    u[lin3(i + 1, j, k, ni + 1, nj)] = U_in;
    v[lin3(i, j, k, ni, nj + 1)] = 0.0f;
    v[lin3(i, j + 1, k, ni, nj + 1)] = 0.0f;
    w[lin3(i, j, k, ni, nj)] = 0.0f;
    w[lin3(i, j, k + 1, ni, nj)] = 0.0f;
  }
}

// Matrix-free assembly, Smoke_solver3D.cpp:984-1111, for interior cells
// 1..n-2 (ring rows stay empty: diag = 0, which the smoother maps to x = 0,
// i.e. Dirichlet p = 0 on the ring).  Writes the FP64 operator (diag, +x,
// +y, +z; the -x/-y/-z couplings the reference also stores are the +x/+y/+z
// couplings of the neighbour, equal by construction) and the FP64 rhs.
// variant 0: SmokeSolver3D::pcg_projection; variant 1:
// SubDomainSolver::pcg_projection (sub_domain.cpp:560-729): the operator
// terms carry the time step, w*dt/h^2, and the solid term is scaled by the
// float 1/h instead of the double 1.0/h.
__global__ void assemble_kernel(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                                const float* __restrict__ uw, const float* __restrict__ vw,
                                const float* __restrict__ ww, const float* __restrict__ us,
                                const float* __restrict__ vs, const float* __restrict__ ws, double* __restrict__ diag,
                                double* __restrict__ xp, double* __restrict__ yp, double* __restrict__ zp,
                                double* __restrict__ rhs, float h, int ni, int nj, int nk, int variant, float dt,
                                float inv_h, float* __restrict__ op32) {
  const size_t n = (size_t)ni * nj * nk;
  const float h2 = h * h;
  // x / h and x / h^2 as products when h is a power of two (inv_h != 0):
  // the same correctly rounded quotients without the division sequence
  const float inv_h2 = inv_h * inv_h;
  auto div_h = [&](float x) { return inv_h != 0.0f ? x * inv_h : x / h; };
  auto div_h2 = [&](float x) { return inv_h != 0.0f ? x * inv_h2 : x / h2; };
  // two cells per thread and round, so each thread has both cells' loads in
  // flight at once (the loop was bound by memory latency)
  auto cell = [&](size_t e) {
    int i, j, k;
    decode3(e, ni, nj, i, j, k);
    double d = 0.0, cx = 0.0, cy = 0.0, cz = 0.0, b = 0.0;
    if (i >= 1 && i < ni - 1 && j >= 1 && j < nj - 1 && k >= 1 && k < nk - 1) {
      const size_t iu0 = lin3(i, j, k, ni + 1, nj), iu1 = lin3(i + 1, j, k, ni + 1, nj);
      const size_t iv0 = lin3(i, j, k, ni, nj + 1), iv1 = lin3(i, j + 1, k, ni, nj + 1);
      const size_t iw0 = lin3(i, j, k, ni, nj), iw1 = lin3(i, j, k + 1, ni, nj);
      const bool sub = variant == 1;
      auto term = [&](float wgt) { return sub ? div_h2(wgt * dt) : div_h2(wgt); };
      // every load up front (one round of memory latency; the solid
      // velocities are read whether or not the cell turns out fluid)
      const float uw1 = uw[iu1], uw0 = uw[iu0], vw1 = vw[iv1], vw0 = vw[iv0], ww1 = ww[iw1], ww0 = ww[iw0];
      const float u1 = u[iu1], u0 = u[iu0], v1 = v[iv1], v0 = v[iv0], w1 = w[iw1], w0 = w[iw0];
      const float us1 = us[iu1], us0 = us[iu0], vs1 = vs[iv1], vs0 = vs[iv0], ws1 = ws[iw1], ws0 = ws[iw0];
      float t;
      t = term(uw1); d = (double)t; if (i < ni - 2) cx = (double)(-t);
      b = b - (double)div_h(uw1 * u1);
      t = term(uw0); d = d + (double)t;
      b = b + (double)div_h(uw0 * u0);
      t = term(vw1); d = d + (double)t; if (j < nj - 2) cy = (double)(-t);
      b = b - (double)div_h(vw1 * v1);
      t = term(vw0); d = d + (double)t;
      b = b + (double)div_h(vw0 * v0);
      t = term(ww1); d = d + (double)t; if (k < nk - 2) cz = (double)(-t);
      b = b - (double)div_h(ww1 * w1);
      t = term(ww0); d = d + (double)t;
      b = b + (double)div_h(ww0 * w0);
      if (d > 0) {
        float sv = (uw1 - 1.0f) * us1 - (uw0 - 1.0f) * us0 + (vw1 - 1.0f) * vs1 -
                   (vw0 - 1.0f) * vs0 + (ww1 - 1.0f) * ws1 - (ww0 - 1.0f) * ws0;
        if (sub) b = b + (double)((1.0f / h) * sv);
        else b = b + (1.0 / (double)h) * (double)sv;
      }
    }
    diag[e] = d;
    xp[e] = cx;
    yp[e] = cy;
    zp[e] = cz;
    rhs[e] = b;
    if (op32) {  // the FP32 copy convert4_kernel would make: [diag | xp | yp | zp]
      op32[e] = (float)d;
      op32[n + e] = (float)cx;
      op32[2 * n + e] = (float)cy;
      op32[3 * n + e] = (float)cz;
    }
  };
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += 2 * stride) {
    cell(e);
    if (e + stride < n) cell(e + stride);
  }
}

// Gradient update, Smoke_solver3D.cpp:1126-1200: on the faces strictly
// between two interior cells (u: i in [2, ni-2], j,k in [1, n-2]; v, w
// analogous) u -= (float)(p_i - p_{i-1}) / h where the face is open, else
// u = u_solid.  Other faces are left untouched, as in the reference.
// variant 1 (SubDomainSolver::pcg_projection, sub_domain.cpp:741-818):
// faces i in [1, ni-1] (all faces between cells of the grid) and
// u -= dt * (float)(p_i - p_{i-1}) / h.
// One thread per cell (i, j, k) updates the three faces with that index
// (u(i,j,k), v(i,j,k), w(i,j,k)): every face the update touches has an index
// inside the cell range, the cell's own pressure is read once for all three,
// and the neighbours' (i-1, j-1, k-1) come from the lines the adjacent
// threads, rows and planes just read.  A face's solid velocity is read only
// where its weight is not positive and its velocity only where it is.
template <typename P>
__global__ void gradient3_kernel(const P* __restrict__ p, float* __restrict__ u, float* __restrict__ v,
                                 float* __restrict__ w, const float* __restrict__ uw, const float* __restrict__ vw,
                                 const float* __restrict__ ww, const float* __restrict__ us,
                                 const float* __restrict__ vs, const float* __restrict__ ws, float h, int ni, int nj,
                                 int nk, int variant, float dt, float inv_h) {
  const size_t n = (size_t)ni * nj * nk;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const bool sub = variant == 1;
  const int lo = sub ? 0 : 1;  // first face index excluded: faces > lo
  const int hi = sub ? 0 : 1;  // faces < n - hi
  auto upd = [&](float cur, double pc, double pm) {
    float diff = (float)(pc - pm);
    // x / h as x * (1/h) when h is a power of two (inv_h != 0): the same bits
    const float q = sub ? dt * diff : diff;
    return cur - (inv_h != 0.0f ? q * inv_h : q / h);
  };
  auto cell = [&](size_t c) {
    int i, j, k;
    decode3(c, ni, nj, i, j, k);
    const bool jin = j < nj - 1 && j > 0, kin = k < nk - 1 && k > 0, iin = i < ni - 1 && i > 0;
    const bool fu = kin && jin && i < ni - hi && i > lo;
    const bool fv = kin && j > lo && j < nj - hi && iin;
    const bool fw = k > lo && k < nk - hi && jin && iin;
    if (!(fu || fv || fw)) return;
    const size_t eu = lin3(i, j, k, ni + 1, nj), ev = lin3(i, j, k, ni, nj + 1), ew = c;
    // the weights, velocities and pressures of the three faces in flight at once
    const float wu = fu ? uw[eu] : 0.0f, wv = fv ? vw[ev] : 0.0f, wwt = fw ? ww[ew] : 0.0f;
    const float cu = fu ? u[eu] : 0.0f, cv = fv ? v[ev] : 0.0f, cw = fw ? w[ew] : 0.0f;
    const double pc = (double)p[c];
    const double pu = fu ? (double)p[c - 1] : 0.0, pv = fv ? (double)p[c - sy] : 0.0,
                 pw = fw ? (double)p[c - sz] : 0.0;
    if (fu) u[eu] = wu > 0 ? upd(cu, pc, pu) : us[eu];
    if (fv) v[ev] = wv > 0 ? upd(cv, pc, pv) : vs[ev];
    if (fw) w[ew] = wwt > 0 ? upd(cw, pc, pw) : ws[ew];
  };
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += 2 * stride) {
    cell(c);
    if (c + stride < n) cell(c + stride);
  }
}

}  // namespace vflip
