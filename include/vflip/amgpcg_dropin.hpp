// Header-only drop-in for the reference solver's pressure-solve entry point
//
//   template<class T> bool ivock::AMGPCGSolve(const SparseMatrix<T>& matrix,
//       const std::vector<T>& rhs, std::vector<T>& result, T tolerance_factor,
//       int max_iterations, T& residual_out, int& iterations_out,
//       int ni, int nj, int nk)              (Smoke_Solver/AlgebraicMultigrid.h:189-197)
//
// Include the caller's sparse_matrix.h (which defines ivock::SparseMatrix<T>,
// Smoke_Solver/sparse_matrix.h:13-192) and then this header INSTEAD OF
// AlgebraicMultigrid.h; SmokeSolver3D::pcg_projection
// (Smoke_solver3D.cpp:1120) and SubDomainSolver::pcg_projection
// (sub_domain.cpp:739) then compile unchanged and solve on the GPU through
// vflip_amgpcg_solve_csr (include/vflip.h).  Link with -lvflip_gpu.
//
// Semantics kept: result is zeroed and written, rhs is read only, the return
// value is the reference's bool (true: |r|_inf <= tolerance_factor *
// |rhs|_inf), residual_out is the absolute inf-norm of the final residual and
// iterations_out the PCG iteration count.  By default the GPU solves in FP64
// (its V-cycle reproduces the reference's bit for bit);
// vflip_dropin::set_precision(VFLIP_PREC_FP32) trades that for speed.  A CUDA
// or argument error (for example a matrix that is not the 7-point symmetric
// operator of the ni x nj x nk grid) prints one line to stderr and returns
// false, as the reference reports a failed solve.
#ifndef VFLIP_AMGPCG_DROPIN_HPP
#define VFLIP_AMGPCG_DROPIN_HPP

#include <cstdint>
#include <cstdio>
#include <vector>

#include "../vflip.h"

namespace vflip_dropin {

inline int& precision_setting() {
  static int p = VFLIP_PREC_FP64;
  return p;
}

inline void set_precision(int precision) { precision_setting() = precision; }

// One context per host thread, created on first use with the reference's
// smoother settings (V(4,4), 200 coarsest sweeps, coarsest <= 16^3).
struct ThreadContext {
  vflip_ctx* ctx = nullptr;
  int precision = -1;
  ~ThreadContext() {
    if (ctx) vflip_destroy(ctx);
  }
  vflip_ctx* get() {
    if (ctx && precision == precision_setting()) return ctx;
    if (ctx) vflip_destroy(ctx);
    ctx = nullptr;
    if (vflip_config_size() != sizeof(vflip_config)) {  // a library built from another vflip.h
      std::fprintf(stderr, "vflip: libvflip_gpu.so was built from another vflip.h (config %zu vs %zu bytes)\n",
                   vflip_config_size(), sizeof(vflip_config));
      return nullptr;
    }
    vflip_config cfg;
    vflip_config_default(&cfg);
    cfg.precision = precision_setting();
    if (vflip_create(&ctx, &cfg) != VFLIP_OK) ctx = nullptr;
    precision = precision_setting();
    return ctx;
  }
};

inline vflip_ctx* context() {
  thread_local ThreadContext tc;
  return tc.get();
}

}  // namespace vflip_dropin

namespace ivock {

template <class T>
struct SparseMatrix;  // the caller's row-vector matrix (sparse_matrix.h)

template <class T>
bool AMGPCGSolve(const SparseMatrix<T>& matrix, const std::vector<T>& rhs, std::vector<T>& result,
                 T tolerance_factor, int max_iterations, T& residual_out, int& iterations_out, int ni, int nj,
                 int nk) {
  const unsigned n = matrix.n;
  std::vector<uint32_t> rowstart(n + 1, 0);
  for (unsigned r = 0; r < n; ++r) rowstart[r + 1] = rowstart[r] + (uint32_t)matrix.index[r].size();
  std::vector<uint32_t> col(rowstart[n]);
  std::vector<double> val(rowstart[n]);
  for (unsigned r = 0; r < n; ++r)
    for (size_t e = 0; e < matrix.index[r].size(); ++e) {
      col[rowstart[r] + e] = matrix.index[r][e];
      val[rowstart[r] + e] = (double)matrix.value[r][e];
    }
  std::vector<double> b(rhs.begin(), rhs.end()), x(n, 0.0);
  result.assign(n, T(0));
  double res = 0.0;
  int it = 0;
  vflip_ctx* ctx = vflip_dropin::context();
  if (!ctx) {
    std::fprintf(stderr, "vflip: no CUDA context\n");
    iterations_out = 0;
    return false;
  }
  int rc = vflip_amgpcg_solve_csr(ctx, n, rowstart.data(), col.data(), val.data(), b.data(), x.data(),
                                  (double)tolerance_factor, max_iterations, &res, &it, ni, nj, nk);
  if (rc < 0) {
    std::fprintf(stderr, "vflip: %s\n", vflip_last_error(ctx));
    iterations_out = 0;
    return false;
  }
  for (unsigned q = 0; q < n; ++q) result[q] = (T)x[q];
  residual_out = (T)res;
  iterations_out = it;
  return rc == VFLIP_OK;
}

}  // namespace ivock

#endif  // VFLIP_AMGPCG_DROPIN_HPP
