// CPU restatement of the vFLIP hot path: the oracle.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load this library (oracle/liboracle.so),
// and only to compare against.  The product (vflip_b200/, libvflip_gpu.so) never
// links, loads or falls back to it.
//
// Each function restates the reference algorithm in this project's own code
// and cites the reference file:line it follows (paths inside the vFLIP
// project, Smoke_Solver/ abbreviated SS/).  The restatement keeps the
// reference's floating-point types and the order of every sum, so its
// results are bit-identical to the reference's wherever the reference is
// deterministic; tests/test_oracle.py pins that against the reference
// compiled from its own sources (oracle/build_ref.py) and against the golden
// fixtures in tests/golden/.  Build with -ffp-contract=off.
//
// Conventions shared with oracle/ref_harness.cpp and the CUDA library:
//   * linear layout, index = i + ni*(j + nj*k), i fastest;
//   * cell grid ni x nj x nk; u faces (ni+1) x nj x nk; v ni x (nj+1) x nk;
//     w ni x nj x (nk+1); nodal solid phi (ni+1) x (nj+1) x (nk+1);
//   * a 7-point operator is 7 arrays of n doubles, in the order
//     diag, -x, +x, -y, +y, -z, +z (the CSR column order of one row with the
//     diagonal moved first).
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

enum { D = 0, XM = 1, XP = 2, YM = 3, YP = 4, ZM = 5, ZP = 6 };

inline size_t lin(int i, int j, int k, int nx, int ny) {
  return (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)k);
}

struct Stencil {
  int ni = 0, nj = 0, nk = 0;
  size_t n = 0;
  std::vector<double> a;  // 7 * n
  void init(int i, int j, int k) {
    ni = i; nj = j; nk = k;
    n = (size_t)i * j * k;
    a.assign(7 * n, 0.0);
  }
  double& c(int s, size_t r) { return a[(size_t)s * n + r]; }
  double c(int s, size_t r) const { return a[(size_t)s * n + r]; }
};

// Off-diagonal slots in CSR column order (ascending column index):
// -z, -y, -x, +x, +y, +z.  SS/AlgebraicMultigrid.h:44-54 walks a row in this
// order, skipping the diagonal.
const int kOffOrder[6] = {ZM, YM, XM, XP, YP, ZP};

inline bool nb(const Stencil& A, int i, int j, int k, int s, size_t& q) {
  int ii = i, jj = j, kk = k;
  switch (s) {
    case XM: ii--; break; case XP: ii++; break;
    case YM: jj--; break; case YP: jj++; break;
    case ZM: kk--; break; case ZP: kk++; break;
    default: break;
  }
  if (ii < 0 || jj < 0 || kk < 0 || ii >= A.ni || jj >= A.nj || kk >= A.nk) return false;
  q = lin(ii, jj, kk, A.ni, A.nj);
  return true;
}

// levelGen::generateLevelsGalerkinCoarsening, SS/GeometricLevelGen.h:28-71,
// with R and P from levelGen::generateRP, SS/GeometricLevelGen.cpp:41-66
// (R = 1/8 over the up-to-8 children, P = injection) and the two SpGEMMs
// temp = A*P (scale 1), A_c = 0.5*R*temp (SS/sparse_matrix.h:370-405).
// Multiplying by 0.0625 (= 0.5*0.125) is exact, so
//   A_c(I,J) = 0.0625 * sum_{child c of I, ascending} temp(c,J),
//   temp(c,J) = sum_{entries of row c in column order with parent J} A(c,.)
// reproduces the SpGEMM's sums term for term.
void coarsen(const Stencil& A, Stencil& C) {
  int cni = C.ni, cnj = C.nj, cnk = C.nk;
  for (int K = 0; K < cnk; ++K)
    for (int J = 0; J < cnj; ++J)
      for (int I = 0; I < cni; ++I) {
        size_t rc = lin(I, J, K, cni, cnj);
        double acc[7];
        bool have[7] = {false, false, false, false, false, false, false};
        for (int s = 0; s < 7; ++s) acc[s] = 0.0;
        // children in ascending fine index: kk outer, then jj, then ii
        for (int kk = 0; kk <= 1; ++kk)
          for (int jj = 0; jj <= 1; ++jj)
            for (int ii = 0; ii <= 1; ++ii) {
              int fi = 2 * I + ii, fj = 2 * J + jj, fk = 2 * K + kk;
              if (fi >= A.ni || fj >= A.nj || fk >= A.nk) continue;
              size_t rf = lin(fi, fj, fk, A.ni, A.nj);
              // temp row rf: walk the fine row in column order, bucket by parent
              double t[7];
              bool th[7] = {false, false, false, false, false, false, false};
              const int order[7] = {ZM, YM, XM, D, XP, YP, ZP};
              for (int o = 0; o < 7; ++o) {
                int s = order[o];
                size_t q;
                if (s != D && !nb(A, fi, fj, fk, s, q)) continue;
                // coarse column of the entry's column cell
                int ci = fi, cj = fj, ck = fk;
                if (s == XM) ci--; else if (s == XP) ci++;
                else if (s == YM) cj--; else if (s == YP) cj++;
                else if (s == ZM) ck--; else if (s == ZP) ck++;
                int PI = ci / 2, PJ = cj / 2, PK = ck / 2;
                int slot;
                if (PI == I && PJ == J && PK == K) slot = D;
                else if (PI == I - 1) slot = XM; else if (PI == I + 1) slot = XP;
                else if (PJ == J - 1) slot = YM; else if (PJ == J + 1) slot = YP;
                else if (PK == K - 1) slot = ZM; else slot = ZP;
                double v = A.c(s, rf);
                if (!th[slot]) { t[slot] = v; th[slot] = true; }
                else t[slot] += v;
              }
              for (int s = 0; s < 7; ++s) {
                if (!th[s]) continue;
                double v = 0.0625 * t[s];
                if (!have[s]) { acc[s] = v; have[s] = true; }
                else acc[s] += v;
              }
            }
        for (int s = 0; s < 7; ++s) C.c(s, rc) = acc[s];
      }
}

void build_levels(const Stencil& A0, std::vector<Stencil>& L) {
  L.clear();
  L.push_back(A0);
  int ni = A0.ni, nj = A0.nj, nk = A0.nk;
  unsigned unknowns = (unsigned)ni * nj * nk;
  while (unknowns > 16 * 16 * 16) {  // SS/GeometricLevelGen.h:46-58
    ni = (int)std::ceil((float)ni / 2.0);
    nj = (int)std::ceil((float)nj / 2.0);
    nk = (int)std::ceil((float)nk / 2.0);
    unknowns = (unsigned)ni * nj * nk;
    Stencil C;
    C.init(ni, nj, nk);
    coarsen(L.back(), C);
    L.push_back(std::move(C));
  }
}

// ivock::RBGS, SS/AlgebraicMultigrid.h:22-103: colour (i+j+k) odd first,
// then even; off-diagonal sum in CSR column order; x = 0 where diag == 0.
void rbgs(const Stencil& A, const double* b, double* x, int iters) {
  for (int it = 0; it < iters; ++it)
    for (int colour = 1; colour >= 0; --colour)
      for (int k = 0; k < A.nk; ++k)
        for (int j = 0; j < A.nj; ++j)
          for (int i = 0; i < A.ni; ++i) {
            if (((i + j + k) & 1) != colour) continue;
            size_t r = lin(i, j, k, A.ni, A.nj);
            double sum = 0;
            for (int o = 0; o < 6; ++o) {
              size_t q;
              if (!nb(A, i, j, k, kOffOrder[o], q)) continue;
              sum += A.c(kOffOrder[o], r) * x[q];
            }
            double diag = A.c(D, r);
            x[r] = (diag != 0) ? (b[r] - sum) / diag : 0;
          }
}

// restriction, SS/AlgebraicMultigrid.h:105-117: r = b - A x with
// multiply_and_subtract (SS/sparse_matrix.h:460-480, subtracting entry by
// entry in column order, diagonal included), then b_c = R r.
void restrict_residual(const Stencil& A, const double* x, const double* b, const Stencil& C, double* bc) {
  std::vector<double> r(A.n);
  const int order[7] = {ZM, YM, XM, D, XP, YP, ZP};
  for (int k = 0; k < A.nk; ++k)
    for (int j = 0; j < A.nj; ++j)
      for (int i = 0; i < A.ni; ++i) {
        size_t row = lin(i, j, k, A.ni, A.nj);
        double v = b[row];
        for (int o = 0; o < 7; ++o) {
          size_t q = row;
          if (order[o] != D && !nb(A, i, j, k, order[o], q)) continue;
          v -= A.c(order[o], row) * x[q];
        }
        r[row] = v;
      }
  // b_c = R r: multiply() starts at 0 and adds 0.125*r over the children in
  // ascending column order (SS/sparse_matrix.h:356-362, GeometricLevelGen.cpp:51-64)
  for (int K = 0; K < C.nk; ++K)
    for (int J = 0; J < C.nj; ++J)
      for (int I = 0; I < C.ni; ++I) {
        double s = 0;
        for (int kk = 0; kk <= 1; ++kk)
          for (int jj = 0; jj <= 1; ++jj)
            for (int ii = 0; ii <= 1; ++ii) {
              int fi = 2 * I + ii, fj = 2 * J + jj, fk = 2 * K + kk;
              if (fi >= A.ni || fj >= A.nj || fk >= A.nk) continue;
              s += 0.125 * r[lin(fi, fj, fk, A.ni, A.nj)];
            }
        bc[lin(I, J, K, C.ni, C.nj)] = s;
      }
}

// prolongatoin, SS/AlgebraicMultigrid.h:118-129: x_f += P x_c (injection).
void prolong_add(const Stencil& A, const Stencil& C, const double* xc, double* xf) {
  for (int k = 0; k < A.nk; ++k)
    for (int j = 0; j < A.nj; ++j)
      for (int i = 0; i < A.ni; ++i)
        xf[lin(i, j, k, A.ni, A.nj)] += xc[lin(i / 2, j / 2, k / 2, C.ni, C.nj)];
}

// amgVCycle / amgPrecond, SS/AlgebraicMultigrid.h:130-188: V(4,4), 200
// sweeps on the coarsest level, all level vectors start at zero.
void vcycle(const std::vector<Stencil>& L, const double* b, double* x) {
  size_t nl = L.size();
  std::vector<std::vector<double>> xs(nl), bs(nl);
  for (size_t l = 0; l < nl; ++l) { xs[l].assign(L[l].n, 0.0); bs[l].assign(L[l].n, 0.0); }
  std::memcpy(bs[0].data(), b, sizeof(double) * L[0].n);
  for (size_t l = 0; l + 1 < nl; ++l) {
    rbgs(L[l], bs[l].data(), xs[l].data(), 4);
    restrict_residual(L[l], xs[l].data(), bs[l].data(), L[l + 1], bs[l + 1].data());
  }
  rbgs(L[nl - 1], bs[nl - 1].data(), xs[nl - 1].data(), 200);
  for (int l = (int)nl - 2; l >= 0; --l) {
    prolong_add(L[l], L[l + 1], xs[l + 1].data(), xs[l].data());
    rbgs(L[l], bs[l].data(), xs[l].data(), 4);
  }
  std::memcpy(x, xs[0].data(), sizeof(double) * L[0].n);
}

// multiply, SS/sparse_matrix.h:342-366: y = A s, row sum in column order from 0.
void spmv(const Stencil& A, const double* s, double* y) {
  const int order[7] = {ZM, YM, XM, D, XP, YP, ZP};
  for (int k = 0; k < A.nk; ++k)
    for (int j = 0; j < A.nj; ++j)
      for (int i = 0; i < A.ni; ++i) {
        size_t row = lin(i, j, k, A.ni, A.nj);
        double v = 0;
        for (int o = 0; o < 7; ++o) {
          size_t q = row;
          if (order[o] != D && !nb(A, i, j, k, order[o], q)) continue;
          v += A.c(order[o], row) * s[q];
        }
        y[row] = v;
      }
}

// BLAS::dot (serial, index order) and BLAS::abs_max (first strict maximum of
// |x|, NaN never wins), SS/blas_wrapper.h:13-43.
double dot(const std::vector<double>& x, const std::vector<double>& y) {
  double s = 0;
  for (size_t i = 0; i < x.size(); ++i) s += x[i] * y[i];
  return s;
}
double abs_max(const std::vector<double>& x) {
  double m = 0;
  size_t at = 0;
  for (size_t i = 0; i < x.size(); ++i)
    if (std::fabs(x[i]) > m) { m = std::fabs(x[i]); at = i; }
  return x.empty() ? 0.0 : std::fabs(x[at]);
}

// AMGPCGSolve, SS/AlgebraicMultigrid.h:189-301.
int amgpcg(const Stencil& A0, const double* rhs, double* result, double tol_factor, int maxit,
           double* residual_out, int* iterations_out) {
  std::vector<Stencil> L;
  build_levels(A0, L);
  size_t n = A0.n;
  std::vector<double> x(n, 0.0), r(rhs, rhs + n), z(n), s(n);
  double res = abs_max(r);
  *residual_out = res;
  if (res == 0) {
    *iterations_out = 0;
    std::memcpy(result, x.data(), sizeof(double) * n);
    return 1;
  }
  double tol = tol_factor * res;
  vcycle(L, r.data(), z.data());
  double rho = dot(z, r);
  if (rho == 0 || rho != rho) {
    *iterations_out = 0;
    std::memcpy(result, x.data(), sizeof(double) * n);
    return 0;
  }
  s = z;
  int it;
  for (it = 0; it < maxit; ++it) {
    spmv(A0, s.data(), z.data());
    double alpha = rho / dot(s, z);
    for (size_t q = 0; q < n; ++q) x[q] += alpha * s[q];
    for (size_t q = 0; q < n; ++q) r[q] += -alpha * z[q];
    res = abs_max(r);
    *residual_out = res;
    if (res <= tol) {
      *iterations_out = it + 1;
      std::memcpy(result, x.data(), sizeof(double) * n);
      return 1;
    }
    vcycle(L, r.data(), z.data());
    double rho_new = dot(z, r);
    double beta = rho_new / rho;
    for (size_t q = 0; q < n; ++q) z[q] += beta * s[q];
    s.swap(z);
    rho = rho_new;
  }
  *iterations_out = it;
  std::memcpy(result, x.data(), sizeof(double) * n);
  return 0;
}

Stencil from_arrays(int ni, int nj, int nk, const double* st) {
  Stencil A;
  A.init(ni, nj, nk);
  std::memcpy(A.a.data(), st, sizeof(double) * 7 * A.n);
  return A;
}

// fraction_inside, SS/levelset_util.cpp:4-13 (segment) and :23-103 (square).
float frac2(float l, float r) {
  if (l < 0 && r < 0) return 1;
  if (l < 0 && r >= 0) return l / (l - r);
  if (l >= 0 && r < 0) return r / (r - l);
  return 0;
}
void rotate4(float* a) {
  float t = a[0];
  a[0] = a[1]; a[1] = a[2]; a[2] = a[3]; a[3] = t;
}
// The reference's rotation loops (levelset_util.cpp:32,44,91) never end when
// the inside corners (phi <= 0) include exact zeros in some patterns, e.g.
// phi = {0, 0, 1, 1}.  Here each loop is bounded by the four rotations; a
// failed search returns -1 and frac4 re-evaluates with exact zeros moved to
// the smallest positive float.  Wherever the reference terminates, the result
// is the reference's.
float frac4_try(float bl, float br, float tl, float tr) {
  int inside = (bl <= 0) + (tl <= 0) + (br <= 0) + (tr <= 0);
  float q[4] = {bl, br, tr, tl};
  if (inside == 4) return 1;
  if (inside == 3) {
    int n = 0;
    while (q[0] < 0) { if (++n > 4) return -1; rotate4(q); }
    float s0 = 1 - frac2(q[0], q[3]);
    float s1 = 1 - frac2(q[0], q[1]);
    return 1 - 0.5f * s0 * s1;
  }
  if (inside == 2) {
    int n = 0;
    while (q[0] >= 0 || !(q[1] < 0 || q[2] < 0)) { if (++n > 4) return -1; rotate4(q); }
    if (q[1] < 0) return 0.5f * (frac2(q[0], q[3]) + frac2(q[1], q[2]));
    float mid = 0.25f * (q[0] + q[1] + q[2] + q[3]);
    if (mid < 0) {
      float area = 0;
      float s1 = 1 - frac2(q[0], q[3]);
      float s3 = 1 - frac2(q[2], q[3]);
      area += 0.5f * s1 * s3;
      float s2 = 1 - frac2(q[2], q[1]);
      float s0 = 1 - frac2(q[0], q[1]);
      area += 0.5f * s0 * s2;
      return 1 - area;
    }
    float area = 0;
    float s0 = frac2(q[0], q[1]);
    float s1 = frac2(q[0], q[3]);
    area += 0.5f * s0 * s1;
    float s2 = frac2(q[2], q[1]);
    float s3 = frac2(q[2], q[3]);
    area += 0.5f * s2 * s3;
    return area;
  }
  if (inside == 1) {
    int n = 0;
    while (q[0] >= 0) { if (++n > 4) return -1; rotate4(q); }
    float s0 = frac2(q[0], q[3]);
    float s1 = frac2(q[0], q[1]);
    return 0.5f * s0 * s1;
  }
  return 0;
}
inline float nudge_zero(float x) { return x == 0.0f ? 1.17549435e-38f : x; }
float frac4(float bl, float br, float tl, float tr) {
  float f = frac4_try(bl, br, tl, tr);
  if (f < 0) f = frac4_try(nudge_zero(bl), nudge_zero(br), nudge_zero(tl), nudge_zero(tr));
  return f;
}
inline float clamp01(float a) { return a < 0.0f ? 0.0f : (a > 1.0f ? 1.0f : a); }  // SS/util.h:172-177

// SmokeSolver3D::compute_face_weights, SS/Smoke_solver3D.cpp:874-944.
void face_weights(int ni, int nj, int nk, const float* phi, float* uw, float* vw, float* ww) {
  int px = ni + 1, py = nj + 1;
  auto P = [&](int i, int j, int k) { return phi[lin(i, j, k, px, py)]; };
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i <= ni; ++i)
        uw[lin(i, j, k, ni + 1, nj)] =
            clamp01(1 - frac4(P(i, j, k), P(i, j + 1, k), P(i, j, k + 1), P(i, j + 1, k + 1)));
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i < ni; ++i)
        vw[lin(i, j, k, ni, nj + 1)] =
            clamp01(1 - frac4(P(i, j, k), P(i, j, k + 1), P(i + 1, j, k), P(i + 1, j, k + 1)));
  for (int k = 0; k <= nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i)
        ww[lin(i, j, k, ni, nj)] =
            clamp01(1 - frac4(P(i, j, k), P(i, j + 1, k), P(i + 1, j, k), P(i + 1, j + 1, k)));
}

// One trilinear sample of a face/cell grid, Buffer3D::sample_linear and
// Buffer3D::at, SS/fluid_buffer3D.h:205-248: world -> grid in double,
// clamp-to-edge indices, lerps in double, result rounded to float.
struct Grid {
  const float* d;
  int nx, ny, nz;
  double h, ox, oy, oz;
  float at(int i, int j, int k) const {
    i = i < 0 ? 0 : (i > nx - 1 ? nx - 1 : i);
    j = j < 0 ? 0 : (j > ny - 1 ? ny - 1 : j);
    k = k < 0 ? 0 : (k > nz - 1 ? nz - 1 : k);
    return d[lin(i, j, k, nx, ny)];
  }
  static double lerp(double a, double b, double c) { return (1.0 - c) * a + c * b; }
  float sample(double wx, double wy, double wz) const {
    double gx = wx / h + ox, gy = wy / h + oy, gz = wz / h + oz;
    int i = (int)std::floor(gx), j = (int)std::floor(gy), k = (int)std::floor(gz);
    double cx = gx - (double)i, cy = gy - (double)j, cz = gz - (double)k;
    double v1 = lerp(lerp(at(i, j, k), at(i + 1, j, k), cx), lerp(at(i, j + 1, k), at(i + 1, j + 1, k), cx), cy);
    double v2 = lerp(lerp(at(i, j, k + 1), at(i + 1, j, k + 1), cx),
                     lerp(at(i, j + 1, k + 1), at(i + 1, j + 1, k + 1), cx), cy);
    return (float)lerp(v1, v2, cz);
  }
};

struct Particle {  // SS/fluid_particle.h:14-20, 40 bytes
  float pos[3];
  float vel[3];
  float dens, temp;
  int hash_idx, sub_hash_idx;
};
static_assert(sizeof(Particle) == 40, "particle record is 40 bytes");

// SmokeSolver3D::hash_FLIP, SS/Smoke_solver3D.cpp:1337-1343: cell =
// int((pos + 0.5h)/h) per axis (truncation toward zero, float arithmetic).
int hash_cell(const Particle& p, int ni, int nj, int nk, float h) {
  float c = 0.5f * h;
  int ijk[3];
  int n[3] = {ni, nj, nk};
  for (int a = 0; a < 3; ++a) {
    float t = (p.pos[a] + c) / h;
    // the reference converts with a C cast; anything outside (-1, n) or NaN
    // lands outside [0, n) on x86 and is dropped
    if (!(t > -1.0f && t < (float)n[a])) return -1;
    ijk[a] = (int)t;
  }
  return ijk[2] * ni * nj + ijk[1] * ni + ijk[0];
}

inline float tent(float r) {  // SmokeSolver3D::H, SS/Smoke_solver3D.h:217-223
  float res = 0;
  if (r >= -1 && r < 0) res = 1 + r;
  if (r >= 0 && r < 1) res = 1 - r;
  return res;
}

}  // namespace

extern "C" {

int oracle_levels(int ni, int nj, int nk, const double* st0, int max_levels, int* dims_out, double* st_out) {
  std::vector<Stencil> L;
  build_levels(from_arrays(ni, nj, nk, st0), L);
  size_t off = 0;
  for (size_t l = 0; l < L.size() && (int)l < max_levels; ++l) {
    dims_out[3 * l] = L[l].ni; dims_out[3 * l + 1] = L[l].nj; dims_out[3 * l + 2] = L[l].nk;
    if (st_out) {
      std::memcpy(st_out + off, L[l].a.data(), sizeof(double) * 7 * L[l].n);
      off += 7 * L[l].n;
    }
  }
  return (int)L.size();
}

void oracle_rbgs(int ni, int nj, int nk, const double* st, const double* b, double* x, int iters) {
  rbgs(from_arrays(ni, nj, nk, st), b, x, iters);
}

void oracle_vcycle(int ni, int nj, int nk, const double* st, const double* b, double* x) {
  std::vector<Stencil> L;
  build_levels(from_arrays(ni, nj, nk, st), L);
  vcycle(L, b, x);
}

void oracle_spmv(int ni, int nj, int nk, const double* st, const double* s, double* y) {
  spmv(from_arrays(ni, nj, nk, st), s, y);
}

int oracle_amgpcg(int ni, int nj, int nk, const double* st, const double* rhs, double* result, double tol,
                  int maxit, double* residual_out, int* iterations_out) {
  return amgpcg(from_arrays(ni, nj, nk, st), rhs, result, tol, maxit, residual_out, iterations_out);
}

void oracle_fraction_inside4(int n, const float* bl, const float* br, const float* tl, const float* tr,
                             float* out) {
  for (int q = 0; q < n; ++q) out[q] = frac4(bl[q], br[q], tl[q], tr[q]);
}

void oracle_face_weights(int ni, int nj, int nk, float h, const float* phi, float* uw, float* vw, float* ww) {
  (void)h;
  face_weights(ni, nj, nk, phi, uw, vw, ww);
}

}  // extern "C"

namespace {
// variant 0: SmokeSolver3D::pcg_projection, SS/Smoke_solver3D.cpp:945-1202
// (inflow overwrite, w/h^2 terms, double 1.0/h solid term, gradient on faces
// strictly inside the interior, AMGPCG 1e-6 / 50);
// variant 1: SubDomainSolver::pcg_projection, SS/sub_domain.cpp:560-821 (no
// inflow, w*dt/h^2 terms, float 1/h solid term, gradient dt*(dp)/h on every
// face between two cells, AMGPCG with the given tolerance / iterations).
int project_impl(int variant, int ni, int nj, int nk, float h, float dt, float U_in, const float* phi,
                 const int8_t* bdesc, const float* us, const float* vs, const float* ws, float* u, float* v,
                 float* w, double* pressure_out, double* rhs_out, double* st_out, float* uw_out, float* vw_out,
                 float* ww_out, int* iterations_out, double* residual_out, double tol, int maxit) {
  const bool sub = variant == 1;
  size_t n = (size_t)ni * nj * nk;
  size_t nu = (size_t)(ni + 1) * nj * nk, nv = (size_t)ni * (nj + 1) * nk, nw = (size_t)ni * nj * (nk + 1);
  std::vector<float> uw(nu), vw(nv), ww(nw);
  face_weights(ni, nj, nk, phi, uw.data(), vw.data(), ww.data());
  auto U = [&](int i, int j, int k) -> float& { return u[lin(i, j, k, ni + 1, nj)]; };
  auto V = [&](int i, int j, int k) -> float& { return v[lin(i, j, k, ni, nj + 1)]; };
  auto W = [&](int i, int j, int k) -> float& { return w[lin(i, j, k, ni, nj)]; };
  auto UW = [&](int i, int j, int k) { return uw[lin(i, j, k, ni + 1, nj)]; };
  auto VW = [&](int i, int j, int k) { return vw[lin(i, j, k, ni, nj + 1)]; };
  auto WW = [&](int i, int j, int k) { return ww[lin(i, j, k, ni, nj)]; };
  auto US = [&](int i, int j, int k) { return us[lin(i, j, k, ni + 1, nj)]; };
  auto VS = [&](int i, int j, int k) { return vs[lin(i, j, k, ni, nj + 1)]; };
  auto WS = [&](int i, int j, int k) { return ws[lin(i, j, k, ni, nj)]; };
  // inflow overwrite, :964-980 (main domain only)
  for (int k = 0; k < nk && !sub; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i)
        if (bdesc[lin(i, j, k, ni, nj)] == 1) {
          U(i, j, k) = U_in; U(i + 1, j, k) = U_in;
          V(i, j, k) = 0; V(i, j + 1, k) = 0;
          W(i, j, k) = 0; W(i, j, k + 1) = 0;
        }
  // assembly over interior cells, :984-1111
  Stencil A;
  A.init(ni, nj, nk);
  std::vector<double> rhs(n, 0.0);
  float h2 = h * h;  // sqr(_hx), float
  for (int k = 1; k < nk - 1; ++k)
    for (int j = 1; j < nj - 1; ++j)
      for (int i = 1; i < ni - 1; ++i) {
        size_t r = lin(i, j, k, ni, nj);
        double diag;
        double b = 0;
        float t;
        // the subdomain's term is w*dt/sqr(h) (SS/sub_domain.cpp:611), evaluated left to right
        auto term = [&](float wgt) { return sub ? wgt * dt / h2 : wgt / h2; };
        t = term(UW(i + 1, j, k)); diag = t; if (i < ni - 2) A.c(XP, r) = -t;
        b -= UW(i + 1, j, k) * U(i + 1, j, k) / h;
        t = term(UW(i, j, k)); diag += t; if (i >= 2) A.c(XM, r) = -t;
        b += UW(i, j, k) * U(i, j, k) / h;
        t = term(VW(i, j + 1, k)); diag += t; if (j < nj - 2) A.c(YP, r) = -t;
        b -= VW(i, j + 1, k) * V(i, j + 1, k) / h;
        t = term(VW(i, j, k)); diag += t; if (j >= 2) A.c(YM, r) = -t;
        b += VW(i, j, k) * V(i, j, k) / h;
        t = term(WW(i, j, k + 1)); diag += t; if (k < nk - 2) A.c(ZP, r) = -t;
        b -= WW(i, j, k + 1) * W(i, j, k + 1) / h;
        t = term(WW(i, j, k)); diag += t; if (k >= 2) A.c(ZM, r) = -t;
        b += WW(i, j, k) * W(i, j, k) / h;
        A.c(D, r) = diag;
        if (diag > 0) {
          float sv = (UW(i + 1, j, k) - 1.0f) * US(i + 1, j, k) - (UW(i, j, k) - 1.0f) * US(i, j, k) +
                     (VW(i, j + 1, k) - 1.0f) * VS(i, j + 1, k) - (VW(i, j, k) - 1.0f) * VS(i, j, k) +
                     (WW(i, j, k + 1) - 1.0f) * WS(i, j, k + 1) - (WW(i, j, k) - 1.0f) * WS(i, j, k);
          if (sub) b += 1 / h * sv;  // float 1/_hx, SS/sub_domain.cpp:716
          else b += 1.0 / h * sv;
        }
        rhs[r] = b;
      }
  std::vector<double> p(n, 0.0);
  double res = 0;
  int it = 0;
  int ok = amgpcg(A, rhs.data(), p.data(), tol, maxit, &res, &it);  // :1120, SS/sub_domain.cpp:739
  // gradient update, :1126-1200 (SS/sub_domain.cpp:741-818 for the subdomain)
  const int lo = sub ? 1 : 2, hi_i = sub ? ni - 1 : ni - 2, hi_j = sub ? nj - 1 : nj - 2, hi_k = sub ? nk - 1 : nk - 2;
  auto grad = [&](float cur, double pc, double pm) {
    return sub ? cur - dt * (float)(pc - pm) / h : cur - (float)(pc - pm) / h;
  };
  for (int k = 1; k < nk - 1; ++k)
    for (int j = 1; j < nj - 1; ++j)
      for (int i = lo; i <= hi_i; ++i) {
        size_t r = lin(i, j, k, ni, nj);
        if (UW(i, j, k) > 0) U(i, j, k) = grad(U(i, j, k), p[r], p[r - 1]);
        else U(i, j, k) = US(i, j, k);
      }
  for (int k = 1; k < nk - 1; ++k)
    for (int j = lo; j <= hi_j; ++j)
      for (int i = 1; i < ni - 1; ++i) {
        size_t r = lin(i, j, k, ni, nj);
        if (VW(i, j, k) > 0) V(i, j, k) = grad(V(i, j, k), p[r], p[r - ni]);
        else V(i, j, k) = VS(i, j, k);
      }
  for (int k = lo; k <= hi_k; ++k)
    for (int j = 1; j < nj - 1; ++j)
      for (int i = 1; i < ni - 1; ++i) {
        size_t r = lin(i, j, k, ni, nj);
        if (WW(i, j, k) > 0) W(i, j, k) = grad(W(i, j, k), p[r], p[r - (size_t)ni * nj]);
        else W(i, j, k) = WS(i, j, k);
      }
  if (pressure_out) std::memcpy(pressure_out, p.data(), sizeof(double) * n);
  if (rhs_out) std::memcpy(rhs_out, rhs.data(), sizeof(double) * n);
  if (st_out) std::memcpy(st_out, A.a.data(), sizeof(double) * 7 * n);
  if (uw_out) std::memcpy(uw_out, uw.data(), sizeof(float) * nu);
  if (vw_out) std::memcpy(vw_out, vw.data(), sizeof(float) * nv);
  if (ww_out) std::memcpy(ww_out, ww.data(), sizeof(float) * nw);
  if (iterations_out) *iterations_out = it;
  if (residual_out) *residual_out = res;
  return ok;
}
}  // namespace

extern "C" {

// SmokeSolver3D::pcg_projection.  Same argument meaning as ref_project in
// oracle/ref_harness.cpp.
int oracle_project(int ni, int nj, int nk, float h, float U_in, const float* phi, const int8_t* bdesc,
                   const float* us, const float* vs, const float* ws, float* u, float* v, float* w,
                   double* pressure_out, double* rhs_out, double* st_out, float* uw_out, float* vw_out,
                   float* ww_out, int* iterations_out, double* residual_out) {
  return project_impl(0, ni, nj, nk, h, 1.0f, U_in, phi, bdesc, us, vs, ws, u, v, w, pressure_out, rhs_out, st_out,
                      uw_out, vw_out, ww_out, iterations_out, residual_out, 1e-6, 50);
}

// SubDomainSolver::pcg_projection with the given tolerance / iterations (the
// reference uses 1e-9 / 1000).
int oracle_project_subdomain(int ni, int nj, int nk, float h, float dt, const float* phi, const float* us,
                             const float* vs, const float* ws, float* u, float* v, float* w, double* pressure_out,
                             double* rhs_out, double* st_out, int* iterations_out, double* residual_out, double tol,
                             int maxit) {
  return project_impl(1, ni, nj, nk, h, dt, 0.0f, phi, nullptr, us, vs, ws, u, v, w, pressure_out, rhs_out, st_out,
                      nullptr, nullptr, nullptr, iterations_out, residual_out, tol, maxit);
}

// The RK2 midpoint backtrace shared by SubDomainSolver::advect_field
// (SS/sub_domain.cpp:210-222) and SmokeSolver3D::advect_field_cubic_clamp
// (SS/Smoke_solver3D.cpp:682-691): the half step in double, the full step in
// float.
static void rk2_backtrace(const Grid* vel, float dt, float wx, float wy, float wz, float p[3]) {
  float a = vel[0].sample(wx, wy, wz), b = vel[1].sample(wx, wy, wz), c = vel[2].sample(wx, wy, wz);
  const float px = (float)((double)wx - 0.5 * (double)dt * (double)a);
  const float py = (float)((double)wy - 0.5 * (double)dt * (double)b);
  const float pz = (float)((double)wz - 0.5 * (double)dt * (double)c);
  a = vel[0].sample(px, py, pz);
  b = vel[1].sample(px, py, pz);
  c = vel[2].sample(px, py, pz);
  p[0] = wx - dt * a;
  p[1] = wy - dt * b;
  p[2] = wz - dt * c;
}

// SubDomainSolver::advect_field, SS/sub_domain.cpp:191-235 (RK2 midpoint
// backtrace, trilinear sample).  Same arguments as ref_advect_rk2.
void oracle_advect_rk2(int ni, int nj, int nk, float h, float dt, const float* u, const float* v, const float* w,
                       int fnx, int fny, int fnz, double fox, double foy, double foz, const float* field,
                       float* out) {
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid gf{field, fnx, fny, fnz, (double)h, fox, foy, foz};
  for (int k = 0; k < fnz; ++k)
    for (int j = 0; j < fny; ++j)
      for (int i = 0; i < fnx; ++i) {
        const float wx = (float)(((double)(float)i - fox) * (double)h);
        const float wy = (float)(((double)(float)j - foy) * (double)h);
        const float wz = (float)(((double)(float)k - foz) * (double)h);
        float p[3];
        rk2_backtrace(vel, dt, wx, wy, wz, p);
        out[lin(i, j, k, fnx, fny)] = gf.sample(p[0], p[1], p[2]);
      }
}

void oracle_hash(int ni, int nj, int nk, float h, const void* particles, int np, int* cell_out) {
  const Particle* p = (const Particle*)particles;
  for (int q = 0; q < np; ++q) cell_out[q] = hash_cell(p[q], ni, nj, nk, h);
}

// SmokeSolver3D::particle_to_grid, SS/Smoke_solver3D.cpp:1451-1510, over the
// buckets hash_FLIP builds (particles of a cell in ascending index order).
void oracle_p2g(int ni, int nj, int nk, float h, const void* particles, int np, int comp, float* field,
                float* coef) {
  const Particle* p = (const Particle*)particles;
  size_t nc = (size_t)ni * nj * nk;
  std::vector<int> cell(np), start(nc + 1, 0), order(np);
  for (int q = 0; q < np; ++q) {
    cell[q] = hash_cell(p[q], ni, nj, nk, h);
    if (cell[q] >= 0) start[cell[q] + 1]++;
  }
  for (size_t c = 0; c < nc; ++c) start[c + 1] += start[c];
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (int q = 0; q < np; ++q)
    if (cell[q] >= 0) order[fill[cell[q]]++] = q;
  int fx = ni + (comp == 0), fy = nj + (comp == 1), fz = nk + (comp == 2);
  double ox = comp == 0 ? 0.5 : 0.0, oy = comp == 1 ? 0.5 : 0.0, oz = comp == 2 ? 0.5 : 0.0;
  for (int k = 0; k < fz; ++k)
    for (int j = 0; j < fy; ++j)
      for (int i = 0; i < fx; ++i) {
        float gx = (float)(((double)(float)i - ox) * (double)h);
        float gy = (float)(((double)(float)j - oy) * (double)h);
        float gz = (float)(((double)(float)k - oz) * (double)h);
        float tw = 1e-5f, tv = 0;
        for (int dk = -1; dk <= 1; ++dk)
          for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di) {
              int ci = i + di, cj = j + dj, ck = k + dk;
              if (ci < 0 || cj < 0 || ck < 0 || ci >= ni || cj >= nj || ck >= nk) continue;
              size_t c = lin(ci, cj, ck, ni, nj);
              for (int e = start[c]; e < start[c + 1]; ++e) {
                const Particle& pp = p[order[e]];
                float wgt = tent((pp.pos[0] - gx) / h) * tent((pp.pos[1] - gy) / h) * tent((pp.pos[2] - gz) / h);
                tw += wgt;
                tv += wgt * pp.vel[comp];
              }
            }
        coef[lin(i, j, k, fx, fy)] = tw;
        field[lin(i, j, k, fx, fy)] = tv / tw;
      }
}

// SmokeSolver3D::particle_from_grid, SS/Smoke_solver3D.cpp:1398-1406
// (flip_ratio == 1: vel += trilinear(delta)); otherwise the FLIP/PIC blend of
// fluid_particle::interpolate, SS/fluid_particle.h:315-328, in double:
// vel = (1-f)*u_new(pos) + f*(vel + delta(pos)).
void oracle_g2p(int ni, int nj, int nk, float h, void* particles, int np, const float* du, const float* dv,
                const float* dw, const float* un, const float* vn, const float* wn, double flip_ratio) {
  Particle* p = (Particle*)particles;
  Grid g[3] = {{du, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
               {dv, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
               {dw, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  Grid gn[3] = {{un, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                {vn, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                {wn, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  for (int q = 0; q < np; ++q) {
    double x = p[q].pos[0], y = p[q].pos[1], z = p[q].pos[2];
    float d[3] = {g[0].sample(x, y, z), g[1].sample(x, y, z), g[2].sample(x, y, z)};
    if (flip_ratio == 1.0) {
      for (int a = 0; a < 3; ++a) p[q].vel[a] += d[a];
    } else {
      for (int a = 0; a < 3; ++a) {
        float s = gn[a].sample(x, y, z);
        p[q].vel[a] = (float)((1.0 - flip_ratio) * (double)s + flip_ratio * (double)(p[q].vel[a] + d[a]));
      }
    }
  }
}

// SmokeSolver3D::traceRK3, SS/Smoke_solver3D.cpp:144-158, through
// get_velocity (:71-87; the subdomain blend is inactive): c1 = 2/9 dt,
// c2 = 3/9 dt computed in double and rounded to float, and - as the reference
// writes it - c3 = (1 - c1 - c2) dt with c1, c2 already carrying dt.
extern "C++" {
template <class F>
static void trace_rk3_f(F sample, const float pos[3], float dt, float out[3]) {
  const float c1 = (float)(2.0 / 9.0 * (double)dt), c2 = (float)(3.0 / 9.0 * (double)dt);
  const float c3 = (float)((1.0 - (double)c1 - (double)c2) * (double)dt);
  float v1[3], v2[3], v3[3], m1[3], m2[3];
  sample(pos, v1);
  const float half = (float)(0.5 * (double)dt), q3 = (float)(0.75 * (double)dt);
  for (int a = 0; a < 3; ++a) m1[a] = pos[a] + half * v1[a];
  sample(m1, v2);
  for (int a = 0; a < 3; ++a) m2[a] = pos[a] + q3 * v2[a];
  sample(m2, v3);
  for (int a = 0; a < 3; ++a) out[a] = pos[a] + c1 * v1[a] + c2 * v2[a] + c3 * v3[a];
}
}  // extern "C++"

static void trace_rk3(const Grid* vel, const float pos[3], float dt, float out[3]) {
  trace_rk3_f([&](const float x[3], float v[3]) {
    for (int a = 0; a < 3; ++a) v[a] = vel[a].sample(x[0], x[1], x[2]);
  }, pos, dt, out);
}

// Buffer3D::sample_grad, SS/fluid_buffer3D.h:249-257, then normalize
// (SS/vec.h:218-219 with mag = sqrt(mag2) + 1e-6, the square root taken in
// double as the reference's build resolves it): the solid normal of
// SmokeSolver3D::get_solid_normal, SS/Smoke_solver3D.cpp:115-124.
static void solid_normal(const Grid& phi, const float pos[3], float n[3]) {
  const double x = pos[0], y = pos[1], z = pos[2], h = phi.h;
  const float r = phi.sample(x + h, y, z), l = phi.sample(x - h, y, z);
  const float u = phi.sample(x, y + h, z), b = phi.sample(x, y - h, z);
  const float f = phi.sample(x, y, z - h), k = phi.sample(x, y, z + h);
  const float g[3] = {(float)((double)(r - l) / h), (float)((double)(u - b) / h), (float)((double)(k - f) / h)};
  for (int a = 0; a < 3; ++a) n[a] = 0.5f * g[a];
  float m2 = n[0] * n[0];
  m2 += n[1] * n[1];
  m2 += n[2] * n[2];
  const float mag = (float)(std::sqrt((double)m2) + 1e-6);
  for (int a = 0; a < 3; ++a) n[a] /= mag;
}

// The nested subdomain as the main solver's samplers see it (vflip_subdomain's
// layout): an ni x nj x nk grid of spacing h at bmin, its face velocities and
// nodal solid phi.
struct SubDesc {
  int ni, nj, nk;
  float h;
  float bmin[3];
  const float *u, *v, *w, *nodal_phi;
};

// SmokeSolver3D's samplers with the subdomain active
// (SS/Smoke_solver3D.cpp:61-124, SS/sub_domain.cpp:61-105, SS/sub_domain.h:176-213).
struct Nest {
  float bmin[3], bmax[3], h;
  Grid vel[3], phi;
  explicit Nest(const SubDesc& s) : h(s.h) {
    const int n[3] = {s.ni, s.nj, s.nk};
    // SubDomainSolver::init, SS/sub_domain.h:161-175: bmax = bmin + (nx, ny, nz) dx
    for (int a = 0; a < 3; ++a) {
      bmin[a] = s.bmin[a];
      bmax[a] = s.bmin[a] + (float)n[a] * s.h;
    }
    const double hd = s.h;
    vel[0] = {s.u, s.ni + 1, s.nj, s.nk, hd, 0.5, 0.0, 0.0};
    vel[1] = {s.v, s.ni, s.nj + 1, s.nk, hd, 0.0, 0.5, 0.0};
    vel[2] = {s.w, s.ni, s.nj, s.nk + 1, hd, 0.0, 0.0, 0.5};
    phi = {s.nodal_phi, s.ni + 1, s.nj + 1, s.nk + 1, hd, 0.5, 0.5, 0.5};
  }
  // is_in (m = 2) and is_in2 (m = 5), SS/sub_domain.h:176-201: strictly
  // inside [bmin + m h, bmax - m h] on every axis, compared in double
  bool inside(const float p[3], double m) const {
    for (int a = 0; a < 3; ++a)
      if (!((double)p[a] > (double)bmin[a] + m * (double)h && (double)p[a] < (double)bmax[a] - m * (double)h))
        return false;
    return true;
  }
  // get_boundary_coef, SS/sub_domain.cpp:96-105: the distance to the box
  // 5h inside the subdomain (smallest |component| over both corners) over
  // 4h, clamped to [0, 1]; all in float
  float coef(const float p[3]) const {
    const float m5 = 5.0f * h;
    float d1 = std::fabs(p[0] - (bmin[0] + m5)), d2 = std::fabs(p[0] - (bmax[0] - m5));
    for (int a = 1; a < 3; ++a) {
      const float e1 = std::fabs(p[a] - (bmin[a] + m5)), e2 = std::fabs(p[a] - (bmax[a] - m5));
      if (e1 < d1) d1 = e1;
      if (e2 < d2) d2 = e2;
    }
    const float d = d2 < d1 ? d2 : d1;
    const float c = d / (4.0f * h);
    return c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
  }
  // SubDomainSolver::get_velocity, SS/sub_domain.cpp:69-76: samples at pos - bmin
  void sub_velocity(const float p[3], float out[3]) const {
    const float q[3] = {p[0] - bmin[0], p[1] - bmin[1], p[2] - bmin[2]};
    for (int a = 0; a < 3; ++a) out[a] = vel[a].sample(q[0], q[1], q[2]);
  }
};

// SmokeSolver3D::get_velocity, SS/Smoke_solver3D.cpp:71-88: the main grid's
// velocity, blended inside is_in2 as c vel_sub + (1 - c) vel (float)
static void nested_velocity(const Grid* vel, const Nest* nest, const float p[3], float out[3]) {
  for (int a = 0; a < 3; ++a) out[a] = vel[a].sample(p[0], p[1], p[2]);
  if (nest && nest->inside(p, 5.0)) {
    float v2[3];
    nest->sub_velocity(p, v2);
    const float c = nest->coef(p);
    for (int a = 0; a < 3; ++a) out[a] = c * v2[a] + (1.0f - c) * out[a];
  }
}

// get_solid_phi, SS/Smoke_solver3D.cpp:104-111: the subdomain's nodal phi
// at pos - bmin inside is_in, the main grid's elsewhere
static float nested_phi(const Grid& phi, const Nest* nest, const float p[3]) {
  if (nest && nest->inside(p, 2.0))
    return nest->phi.sample(p[0] - nest->bmin[0], p[1] - nest->bmin[1], p[2] - nest->bmin[2]);
  return phi.sample(p[0], p[1], p[2]);
}

// get_solid_normal, SS/Smoke_solver3D.cpp:112-124: the gradient of the
// subdomain's phi at pos - bmin (its own h) inside is_in, then normalised
static void nested_normal(const Grid& phi, const Nest* nest, const float p[3], float n[3]) {
  if (nest && nest->inside(p, 2.0)) {
    const float q[3] = {p[0] - nest->bmin[0], p[1] - nest->bmin[1], p[2] - nest->bmin[2]};
    solid_normal(nest->phi, q, n);
  } else {
    solid_normal(phi, p, n);
  }
}

// SmokeSolver3D::advect_FLIP, SS/Smoke_solver3D.cpp:1407-1449: RK3 through
// the grid velocity, then a particle that ends inside a solid (sampled nodal
// phi < 0) moves out along the solid normal by -phi.  With a subdomain, the
// velocity, phi and normal are the nested samplers above.
static void advect_flip_impl(int ni, int nj, int nk, float h, void* particles, int np, const float* u,
                             const float* v, const float* w, const float* nodal_phi, float dt, const Nest* nest) {
  Particle* p = (Particle*)particles;
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid phi = {nodal_phi, ni + 1, nj + 1, nk + 1, (double)h, 0.5, 0.5, 0.5};
  auto sample = [&](const float x[3], float o[3]) { nested_velocity(vel, nest, x, o); };
  for (int q = 0; q < np; ++q) {
    float pos[3];
    trace_rk3_f(sample, p[q].pos, dt, pos);
    const float ph = nested_phi(phi, nest, pos);
    if (ph < 0) {
      float n[3];
      nested_normal(phi, nest, pos, n);
      for (int a = 0; a < 3; ++a) pos[a] -= ph * n[a];
    }
    for (int a = 0; a < 3; ++a) p[q].pos[a] = pos[a];
  }
}

void oracle_advect_flip(int ni, int nj, int nk, float h, void* particles, int np, const float* u, const float* v,
                        const float* w, const float* nodal_phi, float dt) {
  advect_flip_impl(ni, nj, nk, h, particles, np, u, v, w, nodal_phi, dt, nullptr);
}

void oracle_advect_flip_nested(int ni, int nj, int nk, float h, void* particles, int np, const float* u,
                               const float* v, const float* w, const float* nodal_phi, float dt,
                               const SubDesc* sub) {
  const Nest nest(*sub);
  advect_flip_impl(ni, nj, nk, h, particles, np, u, v, w, nodal_phi, dt, &nest);
}

// Counter-based uniform in [-1, 1) for reseeding: a 32-bit integer mix of
// (seed, cell, slot, axis) - the GPU kernel computes the same integers.
// The reference draws frand(-1, 1) from rand() (SS/Smoke_solver3D.h:36-39),
// the same distribution from a sequential generator no parallel code can
// reproduce.
static uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
static float reseed_uniform(uint32_t seed, uint32_t cell, uint32_t slot, uint32_t axis) {
  const uint32_t r = mix32(mix32(mix32(seed ^ 0x9e3779b9u) + cell) + (slot * 3u + axis));
  return -1.0f + 2.0f * ((float)(r >> 8) * (1.0f / 16777216.0f));
}

// SmokeSolver3D::reorder_FLIP, SS/Smoke_solver3D.cpp:1347-1396, after
// hash_FLIP: cells in (k, j, i) order; a cell with fewer than 8 particles
// keeps them and gains 8 - n new ones at (i, j, k) h + r 0.49 h (r uniform in
// [-1, 1)^3, reseed_uniform) with the grid velocity there
// (get_velocity_self, :89-97), density and temperature 0; 8 or 9 stay; 10 or
// more keep their first 8.  Then particles with sampled solid phi < 0 are
// dropped.  Returns the count written (or -needed when capacity is short).
// With a subdomain the final filter reads the nested solid phi (get_solid_phi);
// new particles still take the main grid's velocity.
static int reorder_flip_impl(int ni, int nj, int nk, float h, const void* particles, int np, const float* u,
                             const float* v, const float* w, const float* nodal_phi, unsigned seed, void* out,
                             int capacity, const Nest* nest) {
  const Particle* p = (const Particle*)particles;
  Particle* o = (Particle*)out;
  const size_t nc = (size_t)ni * nj * nk;
  std::vector<std::vector<int>> bucket(nc);
  for (int q = 0; q < np; ++q) {
    const int c = hash_cell(p[q], ni, nj, nk, h);
    if (c >= 0) bucket[(size_t)c].push_back(q);
  }
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid phi = {nodal_phi, ni + 1, nj + 1, nk + 1, (double)h, 0.5, 0.5, 0.5};
  std::vector<Particle> all;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const size_t c = lin(i, j, k, ni, nj);
        const std::vector<int>& b = bucket[c];
        const int cnt = (int)b.size();
        const int keep = cnt < 10 ? cnt : 8;
        for (int e = 0; e < keep; ++e) all.push_back(p[b[e]]);
        for (int e = cnt; e < 8; ++e) {
          Particle n = {};
          const float base[3] = {(float)i * h, (float)j * h, (float)k * h};
          for (int a = 0; a < 3; ++a)
            n.pos[a] = base[a] + reseed_uniform(seed, (uint32_t)c, (uint32_t)e, (uint32_t)a) * 0.49f * h;
          for (int a = 0; a < 3; ++a) n.vel[a] = vel[a].sample(n.pos[0], n.pos[1], n.pos[2]);
          all.push_back(n);
        }
      }
  int count = 0;
  for (const Particle& q : all) {
    if (nested_phi(phi, nest, q.pos) >= 0) {
      if (count < capacity) o[count] = q;
      ++count;
    }
  }
  return count <= capacity ? count : -count;
}

int oracle_reorder_flip(int ni, int nj, int nk, float h, const void* particles, int np, const float* u,
                        const float* v, const float* w, const float* nodal_phi, unsigned seed, void* out,
                        int capacity) {
  return reorder_flip_impl(ni, nj, nk, h, particles, np, u, v, w, nodal_phi, seed, out, capacity, nullptr);
}

int oracle_reorder_flip_nested(int ni, int nj, int nk, float h, const void* particles, int np, const float* u,
                               const float* v, const float* w, const float* nodal_phi, unsigned seed, void* out,
                               int capacity, const SubDesc* sub) {
  const Nest nest(*sub);
  return reorder_flip_impl(ni, nj, nk, h, particles, np, u, v, w, nodal_phi, seed, out, capacity, &nest);
}

// get_solid_phi with the subdomain active at n positions (xyz triples).
void oracle_solid_phi_nested(int ni, int nj, int nk, float h, const float* nodal_phi, const SubDesc* sub,
                             const float* pos, int n, float* out) {
  const Nest nest(*sub);
  const Grid phi = {nodal_phi, ni + 1, nj + 1, nk + 1, (double)h, 0.5, 0.5, 0.5};
  for (int q = 0; q < n; ++q) out[q] = nested_phi(phi, &nest, pos + 3 * (size_t)q);
}

// SmokeSolver3D::time_step, SS/Smoke_solver3D.cpp:390-398: the particles
// that SubDomainSolver::is_halo (SS/sub_domain.h:202-213) finds strictly
// inside [bmin - dx, bmax + dx] on every axis (float), in order; the caller
// passes dx = 0.5 h of the main grid.  Returns the count (negated, nothing
// beyond capacity written, when it exceeds capacity).
int oracle_halo_select(const void* particles, int np, const SubDesc* sub, float dx, void* out, int capacity) {
  const Nest nest(*sub);
  const Particle* p = (const Particle*)particles;
  Particle* o = (Particle*)out;
  int count = 0;
  for (int q = 0; q < np; ++q) {
    bool in = true;
    for (int a = 0; a < 3; ++a)
      in = in && p[q].pos[a] > nest.bmin[a] - dx && p[q].pos[a] < nest.bmax[a] + dx;
    if (in) {
      if (count < capacity) o[count] = p[q];
      ++count;
    }
  }
  return count <= capacity ? count : -count;
}

// ---- smoke scalars and the grid advection forms of SmokeSolver3D

// Buffer3D::cubic_interp_weights + cubic_interp, SS/fluid_buffer3D.h:22-38,
// as Buffer3D<float>::sample_cubic instantiates them: the fraction arrives
// as a float (T = float), the four weights are formed in float, and the
// weighted sum of the double values is taken in double, left to right.
static double cubic_interp(double vm, double v0, double v1, double v2, double t) {
  const float f = (float)t, f2 = f * f, f3 = f2 * f;
  const float wm = -(float)(1. / 3) * f + 0.5f * f2 - (float)(1. / 6) * f3;
  const float w0 = 1.0f - f2 + 0.5f * (f3 - f);
  const float w1 = f + 0.5f * (f2 - f3);
  const float w2 = (float)(1. / 6) * (f3 - f);
  return (double)wm * vm + (double)w0 * v0 + (double)w1 * v1 + (double)w2 * v2;
}

// Buffer3D::sample_cubic, SS/fluid_buffer3D.h:259-326: sixteen x-rows
// (z outer, y inner) over the clamped 4x4x4 neighbourhood, then y, then z.
static float sample_cubic(const Grid& g, double wx, double wy, double wz) {
  const double gx = wx / g.h + g.ox, gy = wy / g.h + g.oy, gz = wz / g.h + g.oz;
  const int i = (int)std::floor(gx), j = (int)std::floor(gy), k = (int)std::floor(gz);
  const double x = gx - (double)i, y = gy - (double)j, z = gz - (double)k;
  double fz[4];
  for (int c = 0; c < 4; ++c) {
    double fy[4];
    for (int b = 0; b < 4; ++b) {
      const int jj = j - 1 + b, kk = k - 1 + c;
      fy[b] = cubic_interp(g.at(i - 1, jj, kk), g.at(i, jj, kk), g.at(i + 1, jj, kk), g.at(i + 2, jj, kk), x);
    }
    fz[c] = cubic_interp(fy[0], fy[1], fy[2], fy[3], y);
  }
  return (float)cubic_interp(fz[0], fz[1], fz[2], fz[3], z);
}

// The eight nodes around a point (Buffer3D::sample_cube_lerp,
// SS/fluid_buffer3D.h:329-356) reduced to their min and max in the
// reference's nesting order (SS/Smoke_solver3D.cpp:698-699).
static void corner_range(const Grid& g, double wx, double wy, double wz, float& lo, float& hi) {
  const int i = (int)std::floor(wx / g.h + g.ox), j = (int)std::floor(wy / g.h + g.oy);
  const int k = (int)std::floor(wz / g.h + g.oz);
  const float v[8] = {g.at(i, j, k),         g.at(i + 1, j, k),         g.at(i, j + 1, k),
                      g.at(i + 1, j + 1, k), g.at(i, j, k + 1),         g.at(i + 1, j, k + 1),
                      g.at(i, j + 1, k + 1), g.at(i + 1, j + 1, k + 1)};
  lo = v[0];
  hi = v[0];
  for (int c = 1; c < 8; ++c) {
    lo = std::min(lo, v[c]);
    hi = std::max(hi, v[c]);
  }
}

// SmokeSolver3D::advect_field_cubic_clamp, SS/Smoke_solver3D.cpp:657-707:
// RK2 backtrace, cubic sample, replaced by the trilinear sample where it
// reaches or leaves the range of the eight surrounding nodes.  Same
// arguments as oracle_advect_rk2 (the field has the velocity's spacing h).
void oracle_advect_cubic_clamp(int ni, int nj, int nk, float h, float dt, const float* u, const float* v,
                               const float* w, int fnx, int fny, int fnz, double fox, double foy, double foz,
                               const float* field, float* out) {
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid gf{field, fnx, fny, fnz, (double)h, fox, foy, foz};
  for (int k = 0; k < fnz; ++k)
    for (int j = 0; j < fny; ++j)
      for (int i = 0; i < fnx; ++i) {
        const float wx = (float)(((double)(float)i - fox) * (double)h);
        const float wy = (float)(((double)(float)j - foy) * (double)h);
        const float wz = (float)(((double)(float)k - foz) * (double)h);
        float p[3];
        rk2_backtrace(vel, dt, wx, wy, wz, p);
        float lo, hi;
        corner_range(gf, p[0], p[1], p[2], lo, hi);
        const float lin_v = gf.sample(p[0], p[1], p[2]);
        const float cub_v = sample_cubic(gf, p[0], p[1], p[2]);
        out[lin(i, j, k, fnx, fny)] = (cub_v <= lo || cub_v >= hi) ? lin_v : cub_v;
      }
}

// SmokeSolver3D::advect_field, SS/Smoke_solver3D.cpp:564-610: traceRK3 with
// step -dt from each node, then a trilinear sample.  The field has its own
// spacing fh (the density and temperature grids are 2ni x 2nj x 2nk at h/2,
// SS/Smoke_solver3D.h:313-315); node (i,j,k) sits at ((i-fox)fh, ...).
void oracle_advect_rk3(int ni, int nj, int nk, float h, float dt, const float* u, const float* v, const float* w,
                       int fnx, int fny, int fnz, double fh, double fox, double foy, double foz, const float* field,
                       float* out) {
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid gf{field, fnx, fny, fnz, fh, fox, foy, foz};
  for (int k = 0; k < fnz; ++k)
    for (int j = 0; j < fny; ++j)
      for (int i = 0; i < fnx; ++i) {
        const float pos[3] = {(float)(((double)(float)i - fox) * fh), (float)(((double)(float)j - foy) * fh),
                              (float)(((double)(float)k - foz) * fh)};
        float back[3];
        trace_rk3(vel, pos, -dt, back);
        out[lin(i, j, k, fnx, fny)] = gf.sample(back[0], back[1], back[2]);
      }
}

// SmokeSolver3D::gen_heat, SS/Smoke_solver3D.cpp:1624-1650: decay density and
// temperature, then set both inside the source: a vertical cylinder of
// radius r about (cx, cz) (float distance) whose height is |y - cy| <= r/4
// (compared in double).  Node (i,j,k) sits at (i,j,k)*fh in float.
void oracle_gen_heat(int fnx, int fny, int fnz, double fh, float dt, float dens_decay, float temp_decay, float cx,
                     float cy, float cz, float radius, float dens, float heat, float* rho, float* temp) {
  const float hf = (float)fh;
  for (int k = 0; k < fnz; ++k)
    for (int j = 0; j < fny; ++j)
      for (int i = 0; i < fnx; ++i) {
        const size_t q = lin(i, j, k, fnx, fny);
        rho[q] = rho[q] / (1.0f + dens_decay * dt);
        temp[q] = temp[q] / (1.0f + temp_decay * dt);
        const float px = (float)i * hf, py = (float)j * hf, pz = (float)k * hf;
        const float dx = px - cx, dz = pz - cz;
        const float d = std::sqrt(dx * dx + dz * dz);
        if (d <= radius && (double)std::fabs(py - cy) <= 0.25 * (double)radius) {
          rho[q] = dens;
          temp[q] = heat;
        }
      }
}

// SmokeSolver3D::add_smokeforce, SS/Smoke_solver3D.cpp:1652-1668: each
// particle's y velocity gains dt (-alpha rho + beta T), rho and T sampled
// trilinearly from the fnx x fny x fnz grids of spacing fh (offsets 0).
void oracle_add_smokeforce(void* particles, int np, int fnx, int fny, int fnz, double fh, const float* rho,
                           const float* temp, float alpha, float beta, float dt) {
  Particle* p = (Particle*)particles;
  const Grid gr{rho, fnx, fny, fnz, fh, 0.0, 0.0, 0.0}, gt{temp, fnx, fny, fnz, fh, 0.0, 0.0, 0.0};
  for (int q = 0; q < np; ++q) {
    const float r = gr.sample(p[q].pos[0], p[q].pos[1], p[q].pos[2]);
    const float t = gt.sample(p[q].pos[0], p[q].pos[1], p[q].pos[2]);
    const float fy = dt * (-alpha * r + beta * t);
    p[q].vel[0] += 0.0f;  // Vec3f(0, fy, 0) is added to all three components
    p[q].vel[1] += fy;
    p[q].vel[2] += 0.0f;
  }
}

// ---- smoke tracers (SmokeSolver3D::emit_tracers / advect_tracers /
// write_tracers, SS/Smoke_solver3D.h:46-160): float4 records x, y, z, density

// emit_tracers' keep test, SS/Smoke_solver3D.h:52-59: inside [2h, L-2h] on
// every axis (float) and density > 0.01 (compared in double).
static bool tracer_kept(const float* t, float h, float lx, float ly, float lz) {
  const float m = 2 * h;
  return t[0] > m && t[1] > m && t[2] > m && t[0] < lx - m && t[1] < ly - m && t[2] < lz - m && (double)t[3] > 0.01;
}

// Offset of new tracer `slot`: attempt a draws x, y, z uniform in [-r, r)
// from the counter hash and accepts the first point with x^2 + z^2 + y^2 <=
// r^2 (the reference's sum order).  The reference draws from rand() over the
// cube of half-width r + h; a cube that just bounds the sphere gives the
// same uniform law with a higher acceptance rate.  After 64 rejected
// attempts (probability below 1e-20) the centre is used.
static void tracer_offset(uint32_t seed, uint32_t slot, float r, float o[3]) {
  for (uint32_t a = 0; a < 64; ++a) {
    const float x = r * reseed_uniform(seed ^ 0x7f4a7c15u, slot, a, 0);
    const float y = r * reseed_uniform(seed ^ 0x7f4a7c15u, slot, a, 1);
    const float z = r * reseed_uniform(seed ^ 0x7f4a7c15u, slot, a, 2);
    if (x * x + z * z + y * y <= r * r) {
      o[0] = x; o[1] = y; o[2] = z;
      return;
    }
  }
  o[0] = o[1] = o[2] = 0.0f;
}

// SmokeSolver3D::emit_tracers, SS/Smoke_solver3D.h:46-85 (the nested
// subdomain's seeding, :86-96, is not restated): the kept tracers in order,
// then `count` new ones of density 1 about (cx, cy, cz).  Returns the new
// number of tracers, negated when it exceeds `capacity` (nothing written).
int oracle_emit_tracers(const float* tracers, int n, float h, float lx, float ly, float lz, float cx, float cy,
                        float cz, float r, int count, unsigned seed, float* out, int capacity) {
  int m = 0;
  for (int q = 0; q < n; ++q) m += tracer_kept(tracers + 4 * (size_t)q, h, lx, ly, lz);
  if (m + count > capacity) return -(m + count);
  m = 0;
  for (int q = 0; q < n; ++q)
    if (tracer_kept(tracers + 4 * (size_t)q, h, lx, ly, lz)) {
      for (int a = 0; a < 4; ++a) out[4 * (size_t)m + a] = tracers[4 * (size_t)q + a];
      ++m;
    }
  for (int s = 0; s < count; ++s) {
    float o[3];
    tracer_offset(seed, (uint32_t)s, r, o);
    float* t = out + 4 * (size_t)(m + s);
    t[0] = cx + o[0];
    t[1] = cy + o[1];
    t[2] = cz + o[2];
    t[3] = 1.0f;
  }
  return m + count;
}

// Counter-based uniform in [0, 1) (frand(0, 1) of the subdomain's tracer
// seeding): the 24 high bits of the reseeding hash of (seed, cell, slot, axis).
static float unit_uniform(uint32_t seed, uint32_t cell, uint32_t slot, uint32_t axis) {
  const uint32_t r = mix32(mix32(mix32(seed ^ 0x2545f491u) + cell) + (slot * 3u + axis));
  return (float)(r >> 8) * (1.0f / 16777216.0f);
}

// The nested subdomain's tracer seeding of emit_tracers, SS/Smoke_solver3D.h:86-96:
// for each subdomain cell in (k, j, i) order, four candidates at
// bmin + (i, j, k) h_s + r h_s (r uniform in [0, 1)^3, unit_uniform with
// slot 0..3) of density 1, kept where the nested solid phi is in (0, h_s).
// Appends to out[m..] up to capacity; returns the number seeded.
static int seed_sub_tracers(const Grid& phi, const Nest& nest, const SubDesc& sub, unsigned seed, float* out,
                            int m, int capacity) {
  int s = 0;
  for (int k = 0; k < sub.nk; ++k)
    for (int j = 0; j < sub.nj; ++j)
      for (int i = 0; i < sub.ni; ++i) {
        const uint32_t c = (uint32_t)lin(i, j, k, sub.ni, sub.nj);
        const float base[3] = {nest.bmin[0] + (float)i * sub.h, nest.bmin[1] + (float)j * sub.h,
                               nest.bmin[2] + (float)k * sub.h};
        for (uint32_t e = 0; e < 4; ++e) {
          float pos[3];
          for (uint32_t a = 0; a < 3; ++a) pos[a] = base[a] + unit_uniform(seed, c, e, a) * sub.h;
          const float ph = nested_phi(phi, &nest, pos);
          if (ph > 0 && ph < sub.h) {
            if (m + s < capacity) {
              float* t = out + 4 * (size_t)(m + s);
              t[0] = pos[0];
              t[1] = pos[1];
              t[2] = pos[2];
              t[3] = 1.0f;
            }
            ++s;
          }
        }
      }
  return s;
}

// emit_tracers with the subdomain active (SS/Smoke_solver3D.h:46-96): the
// kept tracers, the emitter's `count`, then the subdomain's seeds; the main
// grid's nodal phi (ni x nj x nk cells of spacing h) and the subdomain's
// enter the nested solid phi.  Returns the new number of tracers, negated
// when it exceeds `capacity` (the content is then incomplete).
int oracle_emit_tracers_nested(const float* tracers, int n, float h, float lx, float ly, float lz, float cx,
                               float cy, float cz, float r, int count, unsigned seed, int ni, int nj, int nk,
                               const float* nodal_phi, const SubDesc* sub, float* out, int capacity) {
  const Nest nest(*sub);
  const Grid phi = {nodal_phi, ni + 1, nj + 1, nk + 1, (double)h, 0.5, 0.5, 0.5};
  const int m = oracle_emit_tracers(tracers, n, h, lx, ly, lz, cx, cy, cz, r, count, seed, out, capacity);
  if (m < 0) return m;
  const int s = seed_sub_tracers(phi, nest, *sub, seed, out, m, capacity);
  return m + s <= capacity ? m + s : -(m + s);
}

// SmokeSolver3D::advect_tracers, SS/Smoke_solver3D.h:99-120: traceRK3 with
// step dt, then out of a solid along its normal when the sampled nodal phi
// is <= 0 (advect_FLIP's test is < 0), and the density divided by
// 1 + decay*dt (the product in float, the sum and the quotient in double).
// With a subdomain, the nested velocity, phi and normal.
static void advect_tracers_impl(int ni, int nj, int nk, float h, float* tracers, int n, const float* u,
                                const float* v, const float* w, const float* nodal_phi, float dt, float dens_decay,
                                const Nest* nest) {
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid phi = {nodal_phi, ni + 1, nj + 1, nk + 1, (double)h, 0.5, 0.5, 0.5};
  auto sample = [&](const float x[3], float o[3]) { nested_velocity(vel, nest, x, o); };
  for (int q = 0; q < n; ++q) {
    float* t = tracers + 4 * (size_t)q;
    float pos[3];
    trace_rk3_f(sample, t, dt, pos);
    const float ph = nested_phi(phi, nest, pos);
    if (ph <= 0) {
      float nrm[3];
      nested_normal(phi, nest, pos, nrm);
      for (int a = 0; a < 3; ++a) pos[a] -= ph * nrm[a];
    }
    const float d = (float)((double)t[3] / (1.0 + (double)(dens_decay * dt)));
    t[0] = pos[0];
    t[1] = pos[1];
    t[2] = pos[2];
    t[3] = d;
  }
}

void oracle_advect_tracers(int ni, int nj, int nk, float h, float* tracers, int n, const float* u, const float* v,
                           const float* w, const float* nodal_phi, float dt, float dens_decay) {
  advect_tracers_impl(ni, nj, nk, h, tracers, n, u, v, w, nodal_phi, dt, dens_decay, nullptr);
}

void oracle_advect_tracers_nested(int ni, int nj, int nk, float h, float* tracers, int n, const float* u,
                                  const float* v, const float* w, const float* nodal_phi, float dt, float dens_decay,
                                  const SubDesc* sub) {
  const Nest nest(*sub);
  advect_tracers_impl(ni, nj, nk, h, tracers, n, u, v, w, nodal_phi, dt, dens_decay, &nest);
}

// SmokeSolver3D::write_tracers' records, SS/Smoke_solver3D.h:128-140:
// (x/lx - 0.5, y/lx, z/lx - 0.5, density), the subtraction in double.
void oracle_tracer_records(const float* tracers, int n, float lx, float* out) {
  for (int q = 0; q < n; ++q) {
    const float* t = tracers + 4 * (size_t)q;
    float* o = out + 4 * (size_t)q;
    o[0] = (float)((double)(t[0] / lx) - 0.5);
    o[1] = t[1] / lx;
    o[2] = (float)((double)(t[2] / lx) - 0.5);
    o[3] = t[3];
  }
}

// ---- the nested subdomain's particle transfers (SubDomainSolver,
// SS/sub_domain.cpp, SS/sub_domain.h): an ni x nj x nk grid of spacing h
// whose origin sits at bmin in world space; its samples take pos - bmin
// (float) and its face grids have the main grid's offsets.

// x86's float -> int conversion: INT_MIN when out of range or NaN
static int trunc_x86(float t) { return (t >= -2147483648.0f && t < 2147483648.0f) ? (int)t : INT_MIN; }

// SubDomainSolver::hash_FLIP, SS/sub_domain.cpp:1087-1109: the cell of
// pos - bmin + h/2, truncated and clamped into the grid (every particle is
// hashed).
static int sub_cell(const Particle& p, int ni, int nj, int nk, float h, const float* bmin) {
  const int n[3] = {ni, nj, nk};
  int c[3];
  for (int a = 0; a < 3; ++a) {
    float x = p.pos[a] - bmin[a];
    x = x + 0.5f * h;
    const int t = trunc_x86(x / h);
    c[a] = t < 0 ? 0 : (t > n[a] - 1 ? n[a] - 1 : t);
  }
  return (int)lin(c[0], c[1], c[2], ni, nj);
}

void oracle_sub_hash(int ni, int nj, int nk, float h, float bx, float by, float bz, const void* particles, int np,
                     int* cell_out) {
  const Particle* p = (const Particle*)particles;
  const float bmin[3] = {bx, by, bz};
  for (int q = 0; q < np; ++q) cell_out[q] = sub_cell(p[q], ni, nj, nk, h, bmin);
}

// SubDomainSolver::H, SS/sub_domain.h:65-71
static float sub_tent(float r) {
  float res = 0;
  if (r >= -1 && r < 0) res = 1 + r;
  if (r >= 0 && r < 1) res = 1 - r;
  return res;
}

// SubDomainSolver::particle_to_grid, SS/sub_domain.cpp:1204-1265, with
// determineDist (SS/sub_domain.h:89-103): within 4 cells of the
// subdomain's boundary (min of i, ni-i, j, nj-j, k, nk-k) the tent is 4h
// wide and gathers from the 9^3 neighbouring buckets, elsewhere h and 3^3.
// Buckets in (k, j, i) order, particles in hash order, sum(w) from 1e-5.
void oracle_sub_p2g(int ni, int nj, int nk, float h, float bx, float by, float bz, const void* particles, int np,
                    int comp, float* field, float* coef) {
  const Particle* p = (const Particle*)particles;
  const float bmin[3] = {bx, by, bz};
  const size_t nc = (size_t)ni * nj * nk;
  std::vector<std::vector<int>> bucket(nc);
  for (int q = 0; q < np; ++q) bucket[(size_t)sub_cell(p[q], ni, nj, nk, h, bmin)].push_back(q);
  const int fx = ni + (comp == 0), fy = nj + (comp == 1), fz = nk + (comp == 2);
  const double ox = comp == 0 ? 0.5 : 0.0, oy = comp == 1 ? 0.5 : 0.0, oz = comp == 2 ? 0.5 : 0.0;
  for (int k = 0; k < fz; ++k)
    for (int j = 0; j < fy; ++j)
      for (int i = 0; i < fx; ++i) {
        const float gx = (float)(((double)(float)i - ox) * (double)h);
        const float gy = (float)(((double)(float)j - oy) * (double)h);
        const float gz = (float)(((double)(float)k - oz) * (double)h);
        const int dist = std::min(std::min(std::min(i, ni - i), std::min(j, nj - j)), std::min(k, nk - k));
        const int l = dist <= 4 ? 4 : 1;
        const float hk = dist <= 4 ? (float)(4.0 * (double)h) : h;
        float tw = 1e-5f, tv = 0.0f;
        for (int dk = -l; dk <= l; ++dk)
          for (int dj = -l; dj <= l; ++dj)
            for (int di = -l; di <= l; ++di) {
              const int ci = i + di, cj = j + dj, ck = k + dk;
              if (ci < 0 || ci >= ni || cj < 0 || cj >= nj || ck < 0 || ck >= nk) continue;
              for (int q : bucket[lin(ci, cj, ck, ni, nj)]) {
                const float px = p[q].pos[0] - bx, py = p[q].pos[1] - by, pz = p[q].pos[2] - bz;
                const float wgt = sub_tent((px - gx) / hk) * sub_tent((py - gy) / hk) * sub_tent((pz - gz) / hk);
                tw += wgt;
                tv += wgt * p[q].vel[comp];
              }
            }
        const size_t e = lin(i, j, k, fx, fy);
        coef[e] = tw;
        field[e] = tv / tw;
      }
}

// SubDomainSolver::particle_from_grid, SS/sub_domain.cpp:1161-1178:
// vel += the delta grids sampled at pos - bmin.
void oracle_sub_g2p(int ni, int nj, int nk, float h, float bx, float by, float bz, void* particles, int np,
                    const float* du, const float* dv, const float* dw) {
  Particle* p = (Particle*)particles;
  const Grid d[3] = {{du, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                     {dv, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                     {dw, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  for (int q = 0; q < np; ++q) {
    const float x = p[q].pos[0] - bx, y = p[q].pos[1] - by, z = p[q].pos[2] - bz;
    float s[3];
    for (int a = 0; a < 3; ++a) s[a] = d[a].sample(x, y, z);
    for (int a = 0; a < 3; ++a) p[q].vel[a] += s[a];
  }
}

// SubDomainSolver::hash_FLIP + reorder_FLIP, SS/sub_domain.cpp:1110-1159:
// as the main grid's, over the interior cells (1 .. n-2 on each axis) only,
// new particles at bmin + (i, j, k) h + r 0.49 h with the subdomain's
// velocity, and the final filter on the subdomain's solid phi; r from the
// counter-based generator of oracle_reorder_flip.
int oracle_sub_reorder_flip(int ni, int nj, int nk, float h, float bx, float by, float bz, const void* particles,
                            int np, const float* u, const float* v, const float* w, const float* nodal_phi,
                            unsigned seed, void* out, int capacity) {
  const Particle* p = (const Particle*)particles;
  Particle* o = (Particle*)out;
  const float bmin[3] = {bx, by, bz};
  const size_t nc = (size_t)ni * nj * nk;
  std::vector<std::vector<int>> bucket(nc);
  for (int q = 0; q < np; ++q) bucket[(size_t)sub_cell(p[q], ni, nj, nk, h, bmin)].push_back(q);
  const Grid vel[3] = {{u, ni + 1, nj, nk, (double)h, 0.5, 0.0, 0.0},
                       {v, ni, nj + 1, nk, (double)h, 0.0, 0.5, 0.0},
                       {w, ni, nj, nk + 1, (double)h, 0.0, 0.0, 0.5}};
  const Grid phi = {nodal_phi, ni + 1, nj + 1, nk + 1, (double)h, 0.5, 0.5, 0.5};
  std::vector<Particle> all;
  for (int k = 1; k < nk - 1; ++k)
    for (int j = 1; j < nj - 1; ++j)
      for (int i = 1; i < ni - 1; ++i) {
        const size_t c = lin(i, j, k, ni, nj);
        const std::vector<int>& b = bucket[c];
        const int cnt = (int)b.size();
        const int keep = cnt < 10 ? cnt : 8;
        for (int e = 0; e < keep; ++e) all.push_back(p[b[e]]);
        for (int e = cnt; e < 8; ++e) {
          Particle n = {};
          const float base[3] = {bx + (float)i * h, by + (float)j * h, bz + (float)k * h};
          for (int a = 0; a < 3; ++a)
            n.pos[a] = base[a] + reseed_uniform(seed, (uint32_t)c, (uint32_t)e, (uint32_t)a) * 0.49f * h;
          const float q0 = n.pos[0] - bx, q1 = n.pos[1] - by, q2 = n.pos[2] - bz;
          for (int a = 0; a < 3; ++a) n.vel[a] = vel[a].sample(q0, q1, q2);
          all.push_back(n);
        }
      }
  int count = 0;
  for (const Particle& q : all) {
    if (phi.sample(q.pos[0] - bx, q.pos[1] - by, q.pos[2] - bz) >= 0) {
      if (count < capacity) o[count] = q;
      ++count;
    }
  }
  return count <= capacity ? count : -count;
}

// SmokeSolver3D::getDelta, SS/Smoke_solver3D.cpp:1298-1319.
void oracle_delta(int nx, int ny, int nz, const float* after, const float* before, float* delta) {
  size_t n = (size_t)nx * ny * nz;
  for (size_t q = 0; q < n; ++q) delta[q] = after[q] - before[q];
}

int oracle_particle_size() { return (int)sizeof(Particle); }

// The grid smoke-plume step (vflip_b200/plume.py): RK2 advection of the five
// fields (SubDomainSolver::advect_field), the plume sources (this project's
// grid analogue of SS/Smoke_solver3D.cpp:1624-1668), pcg_projection with no
// inflow and resting solids.  Fields are updated in place; returns the
// solver's bool.
int oracle_smoke_step(int n, float h, float dt, const float* phi, float* u, float* v, float* w, float* rho,
                      float* temp, float cx, float cy, float cz, float radius, float alpha, float beta,
                      int* iterations_out, double* residual_out) {
  size_t nc = (size_t)n * n * n, nu = (size_t)(n + 1) * n * n;
  std::vector<float> u2(nu), v2(nu), w2(nu), rho2(nc), temp2(nc);
  oracle_advect_rk2(n, n, n, h, dt, u, v, w, n + 1, n, n, 0.5, 0, 0, u, u2.data());
  oracle_advect_rk2(n, n, n, h, dt, u, v, w, n, n + 1, n, 0, 0.5, 0, v, v2.data());
  oracle_advect_rk2(n, n, n, h, dt, u, v, w, n, n, n + 1, 0, 0, 0.5, w, w2.data());
  oracle_advect_rk2(n, n, n, h, dt, u, v, w, n, n, n, 0, 0, 0, rho, rho2.data());
  oracle_advect_rk2(n, n, n, h, dt, u, v, w, n, n, n, 0, 0, 0, temp, temp2.data());
  std::memcpy(u, u2.data(), 4 * nu);
  std::memcpy(v, v2.data(), 4 * nu);
  std::memcpy(w, w2.data(), 4 * nu);
  std::memcpy(rho, rho2.data(), 4 * nc);
  std::memcpy(temp, temp2.data(), 4 * nc);
  const float r2 = radius * radius;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        float dx = i * h - cx, dy = j * h - cy, dz = k * h - cz;
        if (dx * dx + dy * dy + dz * dz <= r2) {
          rho[lin(i, j, k, n, n)] = 1.0f;
          temp[lin(i, j, k, n, n)] = 1.0f;
        }
      }
  for (int k = 0; k < n; ++k)
    for (int j = 1; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        size_t c0 = lin(i, j - 1, k, n, n), c1 = lin(i, j, k, n, n);
        float r = 0.5f * (rho[c0] + rho[c1]);
        float t = 0.5f * (temp[c0] + temp[c1]);
        size_t e = lin(i, j, k, n, n + 1);
        v[e] = v[e] + dt * (-alpha * r + beta * t);
      }
  std::vector<int8_t> bdesc(nc, 0);
  std::vector<float> zu(nu, 0.0f);
  return oracle_project(n, n, n, h, 0.0f, phi, bdesc.data(), zu.data(), zu.data(), zu.data(), u, v, w, nullptr,
                        nullptr, nullptr, nullptr, nullptr, nullptr, iterations_out, residual_out);
}
}
