// Builds the projection system the way SmokeSolver3D::pcg_projection does
// (row-vector SparseMatrix, add_to_element in the same order) and solves it
// through the header-only drop-in ivock::AMGPCGSolve.  The SparseMatrix here
// is a minimal stand-in with the reference type's members and add_to_element
// semantics (Smoke_Solver/sparse_matrix.h:13-105), written for this test.
//
// Usage: dropin_main <n> <out.bin>   writes rhs, result (n^3 doubles each),
// then ok, iterations, residual; exit status 0 when the solve ran.
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace ivock {
template <class T>
struct SparseMatrix {
  unsigned int n;
  std::vector<std::vector<unsigned int>> index;
  std::vector<std::vector<T>> value;
  explicit SparseMatrix(unsigned int n_ = 0) : n(n_), index(n_), value(n_) {}
  void add_to_element(unsigned int i, unsigned int j, T inc) {
    unsigned int k = 0;
    for (; k < index[i].size(); ++k) {
      if (index[i][k] == j) { value[i][k] += inc; return; }
      if (index[i][k] > j) {
        index[i].insert(index[i].begin() + k, j);
        value[i].insert(value[i].begin() + k, inc);
        return;
      }
    }
    index[i].push_back(j);
    value[i].push_back(inc);
  }
};
}  // namespace ivock

#include "vflip/amgpcg_dropin.hpp"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const int n = std::atoi(argv[1]);
  const float h = 1.0f / n;
  ivock::SparseMatrix<double> A(n * n * n);
  std::vector<double> rhs(n * n * n, 0.0), p;
  unsigned seed = 12345u;
  auto rnd = [&]() { seed = seed * 1664525u + 1013904223u; return ((seed >> 8) & 0xffff) / 65536.0 - 0.5; };
  for (int k = 1; k < n - 1; ++k)
    for (int j = 1; j < n - 1; ++j)
      for (int i = 1; i < n - 1; ++i) {
        int idx = i + n * j + n * n * k;
        float term = 1.0f / (h * h);
        A.add_to_element(idx, idx, term); if (i < n - 2) A.add_to_element(idx, idx + 1, -term);
        A.add_to_element(idx, idx, term); if (i >= 2) A.add_to_element(idx, idx - 1, -term);
        A.add_to_element(idx, idx, term); if (j < n - 2) A.add_to_element(idx, idx + n, -term);
        A.add_to_element(idx, idx, term); if (j >= 2) A.add_to_element(idx, idx - n, -term);
        A.add_to_element(idx, idx, term); if (k < n - 2) A.add_to_element(idx, idx + n * n, -term);
        A.add_to_element(idx, idx, term); if (k >= 2) A.add_to_element(idx, idx - n * n, -term);
        rhs[idx] = rnd();
      }
  double residual = 0;
  int iterations = 0;
  bool ok = ivock::AMGPCGSolve(A, rhs, p, 1e-6, 50, residual, iterations, n, n, n);
  FILE* f = std::fopen(argv[2], "wb");
  if (!f) return 3;
  std::fwrite(rhs.data(), sizeof(double), rhs.size(), f);
  std::fwrite(p.data(), sizeof(double), p.size(), f);
  double tail[3] = {ok ? 1.0 : 0.0, (double)iterations, residual};
  std::fwrite(tail, sizeof(double), 3, f);
  std::fclose(f);
  std::printf("ok=%d iterations=%d residual=%g\n", (int)ok, iterations, residual);
  return 0;
}
