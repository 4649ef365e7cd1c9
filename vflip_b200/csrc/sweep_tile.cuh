// One fused red-black sweep (both colours, out of place) as independent 3-D
// tiles, for the small coarse levels that live in L2.
//
// The plane-marching smoothers pipeline planes through shared memory: right
// for levels that stream from HBM, but a small level then spends its time
// in the march's per-plane latency (a 32^3 level: one row per CTA, ten plane
// steps of about a microsecond each).  Here a CTA owns a TX x TY x TZ tile,
// loads x, b and the operator over the tile and a two-cell halo into shared
// memory at once (from L2), runs the red pass over the tile and a one-cell
// ring, then the black pass over the tile, and stores the tile: two CTA
// barriers per sweep, no march.  The halo is recomputed by neighbouring
// tiles, so no CTA reads a value another writes.
//
// Same values as the other smoothers bit for bit: colour 1 first, then 0;
// the row sum over -z, -y, -x, +x, +y, +z with gs_madd, neighbours outside
// the level skipped (the carry kernel adds them as +-0); (b - sum) / diag
// with gs_div, 0 where diag is 0; ZERO: x_in = 0; PROLONG: x_in + P x_c
// (injection) formed as the values are staged.
#pragma once
#include "common.cuh"

namespace vflip {

constexpr int kTileTX = 16, kTileTY = 8, kTileTZ = 4;
constexpr int kTileRX = kTileTX + 4, kTileRY = kTileTY + 4, kTileRZ = kTileTZ + 4;
constexpr int kTileRegion = kTileRX * kTileRY * kTileRZ;
constexpr int kTileThreads = 256;

template <typename S, typename V>
struct SweepTileArgs {
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
  int ntx, nty;  // tiles along x and y (blockIdx.x = tile index)
};

template <typename S, typename V, bool ZERO, bool PROLONG>
__global__ void __launch_bounds__(kTileThreads) rbgs_sweep_tile_kernel(const SweepTileArgs<S, V> a) {
  using A = typename Num<V>::Acc;
  __shared__ A xs[kTileRegion], bs[kTileRegion], ds[kTileRegion], xps[kTileRegion], yps[kTileRegion],
      zps[kTileRegion];
  const int ni = a.ni, nj = a.nj, nk = a.nk;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const int t = blockIdx.x;
  const int ti = t % a.ntx, tj = (t / a.ntx) % a.nty, tk = t / (a.ntx * a.nty);
  // region origin: the tile's first cell minus the two-cell halo
  const int oi = ti * kTileTX - 2, oj = tj * kTileTY - 2, ok = tk * kTileTZ - 2;
  // staging: every load of the thread's region cells is issued before the
  // first shared-memory store (one round of L2 latency, not one per cell)
  constexpr int kIt = (kTileRegion + kTileThreads - 1) / kTileThreads;
  A xv[kIt], bv[kIt], dv[kIt], cxv[kIt], cyv[kIt], czv[kIt];
#pragma unroll
  for (int q = 0; q < kIt; ++q) {
    const int e = threadIdx.x + q * kTileThreads;
    const int ri = e % kTileRX, rj = (e / kTileRX) % kTileRY, rk = e / (kTileRX * kTileRY);
    const int i = oi + ri, j = oj + rj, k = ok + rk;
    A x = A(0), bb = A(0), d = A(0), cx = A(0), cy = A(0), cz = A(0);
    if (e < kTileRegion && i >= 0 && i < ni && j >= 0 && j < nj && k >= 0 && k < nk) {
      const size_t g = (size_t)i + sy * j + sz * k;
      if (!ZERO) {
        x = ldv(a.x_in + g);
        if (PROLONG) x = x + ldv(a.xc + lin3(i >> 1, j >> 1, k >> 1, a.cni, a.cnj));
      }
      bb = ldv(a.b + g);
      d = A(ldv(a.diag + g));
      cx = A(ldv(a.xp + g));
      cy = A(ldv(a.yp + g));
      cz = A(ldv(a.zp + g));
    }
    xv[q] = x;
    bv[q] = bb;
    dv[q] = d;
    cxv[q] = cx;
    cyv[q] = cy;
    czv[q] = cz;
  }
#pragma unroll
  for (int q = 0; q < kIt; ++q) {
    const int e = threadIdx.x + q * kTileThreads;
    if (e < kTileRegion) {
      xs[e] = xv[q];
      bs[e] = bv[q];
      ds[e] = dv[q];
      xps[e] = cxv[q];
      yps[e] = cyv[q];
      zps[e] = czv[q];
    }
  }
  __syncthreads();
  constexpr int SY = kTileRX, SZ = kTileRX * kTileRY;
  // one colour over the region cells [lo, hi) on every axis (region coordinates)
  auto pass = [&](int lo_x, int hi_x, int lo_y, int hi_y, int lo_z, int hi_z, int parity) {
    const int wx = hi_x - lo_x, wy = hi_y - lo_y, cnt = wx * wy * (hi_z - lo_z);
    for (int q = threadIdx.x; q < cnt; q += kTileThreads) {
      const int ri = lo_x + q % wx, rj = lo_y + (q / wx) % wy, rk = lo_z + q / (wx * wy);
      const int i = oi + ri, j = oj + rj, k = ok + rk;
      if (i < 0 || i >= ni || j < 0 || j >= nj || k < 0 || k >= nk) continue;
      if (((i + j + k) & 1) != parity) continue;
      const int e = ri + SY * rj + SZ * rk;
      A sum = A(0);
      if (k > 0) sum = gs_madd(sum, zps[e - SZ], xs[e - SZ]);
      if (j > 0) sum = gs_madd(sum, yps[e - SY], xs[e - SY]);
      if (i > 0) sum = gs_madd(sum, xps[e - 1], xs[e - 1]);
      if (i < ni - 1) sum = gs_madd(sum, xps[e], xs[e + 1]);
      if (j < nj - 1) sum = gs_madd(sum, yps[e], xs[e + SY]);
      if (k < nk - 1) sum = gs_madd(sum, zps[e], xs[e + SZ]);
      const A d = ds[e];
      xs[e] = (d != A(0)) ? gs_div(bs[e] - sum, d) : A(0);
    }
  };
  pass(1, kTileRX - 1, 1, kTileRY - 1, 1, kTileRZ - 1, 1);  // red: the tile and a one-cell ring
  __syncthreads();
  pass(2, kTileRX - 2, 2, kTileRY - 2, 2, kTileRZ - 2, 0);  // black: the tile
  __syncthreads();
  constexpr int cnt = kTileTX * kTileTY * kTileTZ;
  for (int q = threadIdx.x; q < cnt; q += kTileThreads) {
    const int ri = 2 + q % kTileTX, rj = 2 + (q / kTileTX) % kTileTY, rk = 2 + q / (kTileTX * kTileTY);
    const int i = oi + ri, j = oj + rj, k = ok + rk;
    if (i >= ni || j >= nj || k >= nk) continue;
    a.x_out[(size_t)i + sy * j + sz * k] = cvt<V>(xs[ri + SY * rj + SZ * rk]);
  }
}

}  // namespace vflip
