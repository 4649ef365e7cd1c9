// 3-D-tiled variant of the fused red-black sweep (FP32 vectors, FP32 or BF16
// operator), same arithmetic and schedule as rbgs_sweep_kernel: red on plane
// p over the tile and a one-cell ring, black on plane p-1 over the tile,
// store plane p-1.
//
// A CTA owns a TX x TY tile of every plane of a plane range.  Each array's
// plane footprint (the tile with a 2-row y halo and a 16-byte x halo, so
// every box starts on a 16-byte boundary) arrives by one 3-D TMA tensor load
// (cp.async.bulk.tensor.3d, no multicast; out-of-range cells are filled with
// zeros and skipped by the boundary tests).  The footprints are small (about
// 2 KB per array and plane), so several CTAs share an SM and each keeps D
// copy groups in flight - the full-row kernel fits one CTA and one group.
//
// Rings (plane q in slot q mod ring): x 4+D planes, b/diag/xp/yp 2+D, zp
// 3+D, coarse x 4+D.  Copy groups: G0 = x(k0-2), x(k0-1), zp(k0-2); then
// H(q) = x(q+1), b/diag/xp/yp(q), zp(q) for q >= k0-1 (group q-k0+2).  Every
// mbarrier wait is bounded; on a timeout the CTA sets *error, drains its own
// copies (bounded) and returns.
#pragma once
#include "common.cuh"
#include "sm100.cuh"

namespace vflip {

constexpr int kT3dMaxDepth = 3;
constexpr int kT3dTX = 32, kT3dTY = 8, kT3dBlock = 256;

template <typename S>
struct T3dMaps {
  CUtensorMap x, b, d, xp, yp, zp, xc;
};

struct T3dArgs {
  float* x_out;
  int ni, nj, nk, cni, cnj;
  int ntx;    // tiles along x: blockIdx.x = tile_y * ntx + tile_x
  int zlen;   // planes per CTA: blockIdx.y = plane range
  int depth;  // copy groups in flight, 1..kT3dMaxDepth
  double* dot_partial;
  int* error;
};

template <typename S, int TX, int TY>
struct T3dGeom {
  static constexpr int HX = 4;                    // x halo of the FP32 arrays (16 B)
  static constexpr int HC = 16 / (int)sizeof(S);  // x halo of the coefficient arrays (16 B)
  static constexpr int WX = TX + 2 * HX;          // x, b footprint width
  static constexpr int WC = TX + 2 * HC;          // coefficient footprint width
  static constexpr int H = TY + 4;                // rows y0-2 .. y0+TY+1
  static constexpr int WXC = TX / 2 + 8;          // coarse columns from x0/2 - 4
  static constexpr int HCR = TY / 2 + 2;          // coarse rows from y0/2 - 1
  static constexpr unsigned XB = WX * H * 4;      // bytes one box delivers
  static constexpr unsigned CB = WC * H * sizeof(S);
  static constexpr unsigned XCB = WXC * HCR * 4;
  static constexpr unsigned al(unsigned v) { return (v + 127u) / 128u * 128u; }
  static constexpr unsigned XS = al(XB), CS = al(CB), XCS = al(XCB);  // slot strides
};

template <typename S, int TX, int TY>
__host__ __device__ inline size_t t3d_smem_bytes(int D, bool prolong) {
  using G = T3dGeom<S, TX, TY>;
  return (size_t)(4 + D) * G::XS + (size_t)(2 + D) * G::XS + (size_t)3 * (2 + D) * G::CS + (size_t)(3 + D) * G::CS +
         (prolong ? (size_t)(4 + D) * G::XCS : 0);
}

template <typename S, bool ZERO_X, bool PROLONG, bool DOT, int TX, int TY, int BLOCK>
__global__ void __launch_bounds__(BLOCK) rbgs_sweep_t3d_kernel(const __grid_constant__ T3dMaps<S> mp,
                                                               const T3dArgs a) {
  using G = T3dGeom<S, TX, TY>;
  extern __shared__ __align__(128) unsigned char smraw[];
  constexpr int NB = kT3dMaxDepth + 2;  // mbarrier ring
  __shared__ __align__(8) unsigned long long bars[NB];
  __shared__ double red_smem[BLOCK / 32];
  const int tid = threadIdx.x;
  const int ni = a.ni, nj = a.nj, nk = a.nk, D = a.depth;
  const int RX = 4 + D, RC = 2 + D, RZ = 3 + D;
  // byte offsets of the rings
  const unsigned oX = 0, oB = oX + RX * G::XS, oD = oB + RC * G::XS, oXP = oD + RC * G::CS;
  const unsigned oYP = oXP + RC * G::CS, oZP = oYP + RC * G::CS, oXC = oZP + RZ * G::CS;
  const int ttx = blockIdx.x % a.ntx, tty = blockIdx.x / a.ntx;
  const int x0 = ttx * TX, y0 = tty * TY;
  const int k0 = blockIdx.y * a.zlen;
  const int kend = min(nk, k0 + a.zlen);
  const int xs = x0 - G::HX, cxs = x0 - G::HC, ys = y0 - 2;  // footprint origins
  const int xcs = x0 / 2 - 4, ycs = y0 / 2 - 1;              // coarse footprint origin
  auto X = [&](unsigned off) { return reinterpret_cast<float*>(smraw + off); };
  auto C = [&](unsigned off) { return reinterpret_cast<const S*>(smraw + off); };

  const unsigned sbase = smem_u32(smraw);
  const unsigned bar_base = smem_u32(&bars[0]);
  if (tid == 0) {
    for (int q = 0; q < NB; ++q) mbar_init(bar_base + 8u * q, 1);
    mbar_init_fence();
  }
  __syncthreads();

  auto wrap = [](int v, int r) { return v >= r ? v - r : (v < 0 ? v + r : v); };
  const int p0 = k0 - 1;
  int px = ((p0 % RX) + RX) % RX, pc = ((p0 % RC) + RC) % RC, pz = ((p0 % RZ) + RZ) % RZ;

  // thread 0: copy group g (mbarrier g % NB): x planes qx0/qx1 into x slots
  // sx0/sx1 (and their coarse planes), b/diag/xp/yp plane qc into slot sc,
  // zp plane qz into slot szs; planes outside the domain are skipped
  auto issue = [&](int g, int qx0, int sx0, int qx1, int sx1, int qc, int sc, int qz, int szs) {
    const unsigned bar = bar_base + 8u * (unsigned)(g % NB);
    const bool hx0 = !ZERO_X && qx0 >= 0 && qx0 < nk, hx1 = !ZERO_X && qx1 >= 0 && qx1 < nk;
    const bool hc = qc >= 0 && qc < nk, hz = qz >= 0 && qz < nk;
    const unsigned xb = G::XB + (PROLONG ? G::XCB : 0);
    const unsigned bytes = (hx0 ? xb : 0) + (hx1 ? xb : 0) + (hc ? G::XB + 3 * G::CB : 0) + (hz ? G::CB : 0);
    fence_proxy_async();
    mbar_expect_tx(bar, bytes);
    for (int h = 0; h < 2; ++h) {
      const int qx = h ? qx1 : qx0, sx = h ? sx1 : sx0;
      if (!(h ? hx1 : hx0)) continue;
      tma_tile_3d(sbase + oX + sx * G::XS, &mp.x, xs, ys, qx, bar);
      if (PROLONG) tma_tile_3d(sbase + oXC + sx * G::XCS, &mp.xc, xcs, ycs, qx >> 1, bar);
    }
    if (hc) {
      tma_tile_3d(sbase + oB + sc * G::XS, &mp.b, xs, ys, qc, bar);
      tma_tile_3d(sbase + oD + sc * G::CS, &mp.d, cxs, ys, qc, bar);
      tma_tile_3d(sbase + oXP + sc * G::CS, &mp.xp, cxs, ys, qc, bar);
      tma_tile_3d(sbase + oYP + sc * G::CS, &mp.yp, cxs, ys, qc, bar);
    }
    if (hz) tma_tile_3d(sbase + oZP + szs * G::CS, &mp.zp, cxs, ys, qz, bar);
  };
  auto wait_group = [&](int g) -> bool {
    const bool ok = mbar_wait_bounded(bar_base + 8u * (unsigned)(g % NB), (unsigned)((g / NB) & 1));
    return __syncthreads_and(ok) != 0;
  };

  // relax colour `odd` of plane p on rows [r0, r1) x columns [c0, c1):
  // row sum in the reference's column order (-z, -y, -x, +x, +y, +z), then
  // (b - sum) / diag
  auto relax = [&](int p, int odd, int r0, int r1, int c0, int c1, unsigned sx0, unsigned sxm, unsigned sxp,
                   unsigned sb, unsigned sd, unsigned sxq, unsigned syq, unsigned szq, unsigned szm) {
    const bool zlo = p > 0, zhi = p < nk - 1;
    const int half = (c1 - c0 + 1) >> 1, nrow = r1 - r0;
    float* x = X(sx0);
    const float* xm = X(sxm);
    const float* xq = X(sxp);
    const float* bb = X(sb);
    const S* dd = C(sd);
    const S* cx = C(sxq);
    const S* cy = C(syq);
    const S* cz = C(szq);
    const S* czm = C(szm);
    for (int e = tid; e < nrow * half; e += BLOCK) {
      const int jr = e / half, m = e - jr * half;
      const int j = r0 + jr;
      const int i = c0 + ((c0 + j + p + odd) & 1) + 2 * m;
      if (i >= c1) continue;
      const int fy = j - ys;
      const int s = fy * G::WX + (i - xs), c = fy * G::WC + (i - cxs);
      float sum = 0.0f;
      if (zlo) sum = gs_madd(sum, float(ldv(czm + c)), xm[s]);
      if (j > 0) sum = gs_madd(sum, float(ldv(cy + c - G::WC)), x[s - G::WX]);
      if (i > 0) sum = gs_madd(sum, float(ldv(cx + c - 1)), x[s - 1]);
      if (i < ni - 1) sum = gs_madd(sum, float(ldv(cx + c)), x[s + 1]);
      if (j < nj - 1) sum = gs_madd(sum, float(ldv(cy + c)), x[s + G::WX]);
      if (zhi) sum = gs_madd(sum, float(ldv(cz + c)), xq[s]);
      const float dv = float(ldv(dd + c));
      x[s] = (dv != 0.0f) ? gs_div(bb[s] - sum, dv) : 0.0f;
    }
  };
  auto prolong_add = [&](int q, int slot) {
    if (q < 0 || q >= nk) return;
    float* x = X(oX + slot * G::XS);
    const float* xc = X(oXC + slot * G::XCS);
    for (int e = tid; e < G::WX * G::H; e += BLOCK) {
      const int fy = e / G::WX, fx = e - fy * G::WX;
      const int ci = ((xs + fx) >> 1) - xcs, cj = ((ys + fy) >> 1) - ycs;
      x[e] = x[e] + xc[cj * G::WXC + ci];
    }
  };
  auto zero_x = [&](int slot) {
    float* x = X(oX + slot * G::XS);
    for (int e = tid; e < G::WX * G::H; e += BLOCK) x[e] = 0.0f;
  };

  const int rr0 = max(y0 - 1, 0), rr1 = min(y0 + TY + 1, nj), rc0 = max(x0 - 1, 0), rc1 = min(x0 + TX + 1, ni);
  const int br1 = min(y0 + TY, nj), bc1 = min(x0 + TX, ni);
  double dot = 0.0;
  bool failed = false;
  int issued = 1;
  if (tid == 0) issue(0, p0 - 1, wrap(px - 1, RX), p0, px, -1, 0, p0 - 1, wrap(pz - 1, RZ));
  for (int d = 0; d < D && p0 + d <= kend; ++d) {
    if (tid == 0)
      issue(1 + d, p0 + d + 1, wrap(px + d + 1, RX), -1, 0, p0 + d, wrap(pc + d, RC), p0 + d, wrap(pz + d, RZ));
    issued = 2 + d;
  }
  for (int p = p0; p <= kend; ++p) {
    if (p == p0 && !wait_group(0)) {
      failed = true;
      break;
    }
    if (!wait_group(p - k0 + 2)) {
      failed = true;
      break;
    }
    if (p + D <= kend) {
      if (tid == 0)
        issue(p + D - k0 + 2, p + D + 1, wrap(px + D + 1, RX), -1, 0, p + D, wrap(pc + D, RC), p + D,
              wrap(pz + D, RZ));
      issued = p + D - k0 + 3;
    }
    const int sxm2 = wrap(px - 2, RX), sxm1 = wrap(px - 1, RX), sxp1 = wrap(px + 1, RX);
    const int scm1 = wrap(pc - 1, RC);
    const int szm2 = wrap(pz - 2, RZ), szm1 = wrap(pz - 1, RZ);
    if (PROLONG || ZERO_X) {
      if (p == p0) {
        if (PROLONG) {
          prolong_add(p - 1, sxm1);
          prolong_add(p, px);
        }
        if (ZERO_X) {
          zero_x(sxm1);
          zero_x(px);
        }
      }
      if (PROLONG) prolong_add(p + 1, sxp1);
      if (ZERO_X) zero_x(sxp1);
      __syncthreads();
    }
    if (p >= 0 && p < nk)
      relax(p, 1, rr0, rr1, rc0, rc1, oX + px * G::XS, oX + sxm1 * G::XS, oX + sxp1 * G::XS, oB + pc * G::XS,
            oD + pc * G::CS, oXP + pc * G::CS, oYP + pc * G::CS, oZP + pz * G::CS, oZP + szm1 * G::CS);
    __syncthreads();
    const int q = p - 1;
    const bool out_plane = (q >= k0 && q < kend);
    if (out_plane)
      relax(q, 0, y0, br1, x0, bc1, oX + sxm1 * G::XS, oX + sxm2 * G::XS, oX + px * G::XS, oB + scm1 * G::XS,
            oD + scm1 * G::CS, oXP + scm1 * G::CS, oYP + scm1 * G::CS, oZP + szm1 * G::CS, oZP + szm2 * G::CS);
    __syncthreads();
    if (out_plane) {
      const float* xsrc = X(oX + sxm1 * G::XS);
      const float* bsrc = X(oB + scm1 * G::XS);
      const size_t plane = (size_t)q * ni * nj;
      const int ncol = bc1 - x0, nrow = br1 - y0;
      for (int e = tid; e < nrow * ncol; e += BLOCK) {
        const int r = e / ncol, cidx = e - r * ncol;
        const int s = (y0 + r - ys) * G::WX + (x0 + cidx - xs);
        const float v = xsrc[s];
        a.x_out[plane + (size_t)(y0 + r) * ni + x0 + cidx] = v;
        if (DOT) dot += (double)v * (double)bsrc[s];
      }
    }
    px = wrap(px + 1, RX);
    pc = wrap(pc + 1, RC);
    pz = wrap(pz + 1, RZ);
  }
  if (failed) {
    if (tid == 0) atomicExch(a.error, 1);
    for (int g = max(0, issued - NB); g < issued; ++g)
      mbar_wait_bounded(bar_base + 8u * (unsigned)(g % NB), (unsigned)((g / NB) & 1));
    return;
  }
  if (DOT) {
    double s = block_sum<BLOCK>(dot, red_smem);
    if (tid == 0) a.dot_partial[blockIdx.x + gridDim.x * blockIdx.y] = s;
  }
}

}  // namespace vflip
