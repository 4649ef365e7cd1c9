// Smoke-plume sources and buoyancy for the grid plume scenes.  The
// reference's own sources act on particles and on 2x-refined density /
// temperature grids (SmokeSolver3D::gen_heat / add_smokeforce,
// Smoke_Solver/Smoke_solver3D.cpp:1624-1668, not called by time_step); this
// is their grid analogue: density and temperature are set inside a source
// sphere every step, and the vertical faces receive the buoyancy
// dt * (-alpha * rho + beta * T) averaged from the two cells they separate.
#pragma once
#include "common.cuh"

namespace vflip {

__global__ void plume_sources_kernel(float* __restrict__ rho, float* __restrict__ temp, int ni, int nj, int nk,
                                     float h, float cx, float cy, float cz, float radius, float dens_value,
                                     float heat_value) {
  const size_t nc = (size_t)ni * nj * nk;
  const float r2 = radius * radius;
  // pass 1 (cells): source sphere, cell centre (i,j,k)*h
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nc; e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(e, ni, nj, i, j, k);
    float dx = i * h - cx, dy = j * h - cy, dz = k * h - cz;
    if (dx * dx + dy * dy + dz * dz <= r2) {
      rho[e] = dens_value;
      temp[e] = heat_value;
    }
  }
}

// Buoyancy on interior v faces (between cells j-1 and j); reads the
// post-source density and temperature, so it runs as its own launch.
__global__ void buoyancy_kernel(const float* __restrict__ rho, const float* __restrict__ temp, float* __restrict__ v,
                                int ni, int nj, int nk, float dt, float alpha, float beta) {
  const size_t nv = (size_t)ni * (nj + 1) * nk;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nv; e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    decode3(e, ni, nj + 1, i, j, k);
    if (j < 1 || j >= nj) continue;
    size_t c0 = lin3(i, j - 1, k, ni, nj), c1 = lin3(i, j, k, ni, nj);
    float r = 0.5f * (rho[c0] + rho[c1]);
    float t = 0.5f * (temp[c0] + temp[c1]);
    v[e] = v[e] + dt * (-alpha * r + beta * t);
  }
}

}  // namespace vflip
