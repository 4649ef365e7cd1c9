// Register-carry form of the TMA-pipelined fused red-black sweep.
//
// Same staging (bulk plane copies into the shared-memory rings of
// tma_layout, one copy group in flight, optional L2 prefetch further ahead),
// same schedule (step p: red on plane p over the tile and its one-row ring,
// then black on plane p-1 over the tile and the store) and the same
// per-cell arithmetic (relax_quad_cell) as rbgs_sweep_tma_kernel, so the two
// kernels give bit-identical results.  What changes is who reads what:
//
//   each thread owns ONE quad (four consecutive cells) of ONE row for the
//   whole march along z, and keeps in registers what it loaded or computed
//   for that quad one and two planes back: x of planes p-2 .. p+1 and the
//   coefficients (b, diag, xp, yp, yp of the row below, zp) of planes p-1
//   and p, zp of p-2.  The black pass of plane p-1 then needs from shared
//   memory only the two neighbouring rows (after their red update); the red
//   pass reads the quad's own plane-p coefficients, the next plane of x and
//   the two neighbouring rows.  Left/right neighbours along x come from the
//   adjacent lanes by warp shuffle (shared memory only across a warp edge).
//
// That halves the shared-memory traffic of the relaxation (which bounded the
// plane step: the copies alone run at HBM speed) and removes the 4-way bank
// conflicts of the scalar neighbour loads.
//
// Shape: blockDim = (bx, by) with bx >= quads per row and by >= tile rows +
// 2 (the host checks), so every (row, quad) of the red pass has exactly one
// owner.  Every wait is bounded as in rbgs_sweep_tma_kernel.
//
// NI, TYO, DEPTH (0: read from the arguments) fix the row width, the tile
// rows and the copy depth at compile time; the shared-memory layout's
// offsets then fold into the load addresses (the host launches such an
// instance only for arguments with those values).
#pragma once
#include "mg_kernels.cuh"

namespace vflip {

// Coefficients of one plane of the thread's quad: b, diag, +x, +y, and the
// +y coupling of the row below (its -y coupling).
struct CarryCoef {
  float4 bb, dd, cx, cyp, cym;
};

// relax_quad_cell with every neighbour term present.  A neighbour outside
// the domain enters with x = +0 and a finite coupling, so its term is +-0;
// the row sum starts at +0 and, in round-to-nearest, a sum is -0 only when
// both addends are, so it never becomes -0 and adding +-0 leaves its bits
// unchanged: the same result as skipping the term, without the selects.
template <int K>
__device__ __forceinline__ float relax_quad_cell_m(const float4& xc, const float4& xym, const float4& xyp,
                                                   const float4& xzm, const float4& xzp, float xl, float xr,
                                                   const CarryCoef& C, float cxl, const float4& czp,
                                                   const float4& czm) {
  constexpr int KL = K > 0 ? K - 1 : 0, KR = K < 3 ? K + 1 : 3;
  float sum = 0.0f;
  sum = gs_madd(sum, c4<K>(czm), c4<K>(xzm));
  sum = gs_madd(sum, c4<K>(C.cym), c4<K>(xym));
  sum = gs_madd(sum, (K == 0 ? cxl : c4<KL>(C.cx)), (K == 0 ? xl : c4<KL>(xc)));
  sum = gs_madd(sum, c4<K>(C.cx), (K == 3 ? xr : c4<KR>(xc)));
  sum = gs_madd(sum, c4<K>(C.cyp), c4<K>(xyp));
  sum = gs_madd(sum, c4<K>(czp), c4<K>(xzp));
  const float d = c4<K>(C.dd);
  return (d != 0.0f) ? gs_div(c4<K>(C.bb) - sum, d) : 0.0f;
}

template <typename S, bool ZERO_X, bool PROLONG, bool DOT, int BLOCK, int NI = 0, int TYO = 0, int DEPTH = 0>
__global__ void __launch_bounds__(BLOCK, BLOCK <= 256 ? 2 : 1) rbgs_sweep_carry_kernel(TmaSweepArgs<S> a) {
  extern __shared__ __align__(128) float sm[];
  constexpr int NB = kTmaMaxDepth + 2;
  __shared__ __align__(8) unsigned long long bars[NB];
  __shared__ double red_smem[BLOCK / 32];
  constexpr unsigned FULL = 0xffffffffu;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int ni = NI ? NI : a.ni, nj = a.nj, nk = a.nk, tyo = TYO ? TYO : a.tyo, D = DEPTH ? DEPTH : a.depth;
  const size_t sy = (size_t)ni, sz = (size_t)ni * nj;
  const TmaLayout Ly = tma_layout<S>(ni, tyo, D, PROLONG ? a.crows_max : 0, PROLONG ? a.cni : 0);
  const int xslot = Ly.xslot, cslot = Ly.cslot, yslot = Ly.yslot, cplane = Ly.cplane;
  const int RX = 4 + D, RC = 2 + D, RZ = 3 + D;
  const int oX = Ly.oX, oB = Ly.oB, oXC = Ly.oXC;
  const int oD = Ly.cD, oXP = Ly.cXP, oYP = Ly.cYP, oZP = Ly.cZP;
  const S* cs = reinterpret_cast<const S*>(sm + Ly.oC);
  const unsigned cbase_b = 4u * (unsigned)Ly.oC;
  constexpr unsigned ES = sizeof(S);

  const int j0 = blockIdx.x * tyo;
  const int k0 = blockIdx.y * a.zlen;
  const int kend = min(nk, k0 + a.zlen);
  const int jout1 = min(j0 + tyo, nj);
  const int jr0 = max(j0 - 2, 0), jr1 = min(j0 + tyo + 2, nj);
  const int jred0 = max(j0 - 1, 0), jred1 = min(j0 + tyo + 1, nj);
  const int jy0 = jr0;
  const int xrows = jr1 - jr0, crows = jred1 - jred0, yrows = jred1 - jy0;
  const int cr0 = jr0 >> 1, cr1 = ((jr1 - 1) >> 1) + 1;

  // this thread's quad
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int Q = ni >> 2;
  const int j = jred0 + ty;
  const int i0 = 4 * tx;
  const bool act_red = j < jred1 && tx < Q;                     // red pass: tile + ring rows
  const bool act_blk = act_red && j >= j0 && j < jout1;         // black pass and store: tile rows
  const int xo = (j - jr0) * ni + i0, co = (j - jred0) * ni + i0, yo = (j - jy0) * ni + i0;
  const bool ylo = j > 0, yhi = j < nj - 1;
  const bool xlo = i0 > 0;
  const bool warp_l = (tx & 31) == 0, warp_r = (tx & 31) == 31 || tx + 1 >= Q;
  const bool need_r = tx + 1 < Q;

  const unsigned sbase = smem_u32(sm);
  const unsigned bar_base = smem_u32(&bars[0]);
  if (tid == 0) {
    for (int q = 0; q < NB; ++q) mbar_init(bar_base + 8u * q, 1);
    mbar_init_fence();
  }
  __syncthreads();

  auto wrap = [](int v, int r) { return v >= r ? v - r : (v < 0 ? v + r : v); };
  const int p0 = k0 - 1;
  int px = ((p0 % RX) + RX) % RX, pc = ((p0 % RC) + RC) % RC, pz = ((p0 % RZ) + RZ) % RZ;

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
  auto wait_group = [&](int g) -> bool {
    const bool ok = mbar_wait_bounded(bar_base + 8u * (unsigned)(g % NB), (unsigned)((g / NB) & 1));
    return __syncthreads_and(ok) != 0;
  };
  static_assert(!(ZERO_X && PROLONG), "the prolongation needs an incoming x");
  // PROLONG: the staged x planes hold x_in; x_in + P x_c (injection of the
  // staged coarse plane of the same slot) is formed where an old x value is
  // read - the thread's own quad when it enters the registers, the y and
  // x-edge neighbours of the red pass - and the red pass stores only the red
  // cells, so the shared-memory black cells stay x_in for every reader
  auto cadd4 = [&](float4 v, int slot, int jj) -> float4 {
    if (!PROLONG) return v;
    const float2 c = *reinterpret_cast<const float2*>(sm + oXC + slot * cplane + ((jj >> 1) - cr0) * a.cni +
                                                      (i0 >> 1));
    v.x = v.x + c.x;
    v.y = v.y + c.x;
    v.z = v.z + c.y;
    v.w = v.w + c.y;
    return v;
  };
  auto cadd1 = [&](float v, int slot, int jj, int ii) -> float {
    return PROLONG ? v + sm[oXC + slot * cplane + ((jj >> 1) - cr0) * a.cni + (ii >> 1)] : v;
  };

  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  // ZERO_X without a prolongation: the old x is zero everywhere, so the red
  // pass takes zeros instead of loading them; the red store writes whole
  // quads, so every x the black pass reads from shared memory is written
  // first and the x ring needs no zero fill
  constexpr bool XZ = ZERO_X && !PROLONG;
  // carried state of the thread's quad (see the header comment)
  float4 X2 = z4, X1 = z4, X0 = z4;  // x of p-2, p-1 (red-updated), p
  CarryCoef P{z4, z4, z4, z4, z4};   // coefficients of p-1
  float4 pczp = z4, pczm = z4;       // zp of p-1, p-2
  double dot = 0.0;

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
    // the copy group of plane p+D is issued first thing, so it has the whole
    // step to land
    if (p + D <= kend) {
      if (tid == 0) issue(p + D - k0 + 2, p + D + 1, wrap(px + D + 1, RX), -1, 0, p + D, wrap(pc + D, RC), p + D,
                          wrap(pz + D, RZ));
      issued = p + D - k0 + 3;
    }
    const int sxm1 = wrap(px - 1, RX), sxp1 = wrap(px + 1, RX);
    const int scm1 = wrap(pc - 1, RC);
    const int szm1 = wrap(pz - 1, RZ);
    const int x0 = oX + px * xslot, xm = oX + sxm1 * xslot;
    if (p == p0 && act_red) {
      // entering the march: the planes before p0 come from shared memory
      // (old values; only their black cells are read by red(p0))
      if (!XZ && p >= 1) X1 = cadd4(ld4f(sm + xm + xo), sxm1, j);
      if (!XZ && p >= 0 && p < nk) X0 = cadd4(ld4f(sm + x0 + xo), px, j);
      if (p >= 1) pczp = ld4f(cs + oZP + szm1 * cslot + co);
    }

    // ---- red update of plane p (tile + ring rows)
    const bool do_red = p >= 0 && p < nk;
    // the next plane's x (old values) rides along even when plane p itself
    // is outside the domain (p = -1), so X0 holds x(p) on every entry
    float4 xn = z4, xym = z4, xyp = z4, czp = z4;
    CarryCoef C{z4, z4, z4, z4, z4};
    if (!XZ && act_red && p + 1 >= 0 && p + 1 < nk) xn = cadd4(ld4f(sm + oX + sxp1 * xslot + xo), sxp1, j);
    if (do_red && act_red) {
      if (!XZ && ylo) xym = cadd4(ld4f(sm + x0 + xo - ni), px, j - 1);
      if (!XZ && yhi) xyp = cadd4(ld4f(sm + x0 + xo + ni), px, j + 1);
      C.bb = ld4f(sm + oB + pc * cslot + co);
      C.dd = ld4f(cs + oD + pc * cslot + co);
      C.cx = ld4f(cs + oXP + pc * cslot + co);
      C.cyp = ld4f(cs + oYP + pc * yslot + yo);
      if (ylo) C.cym = ld4f(cs + oYP + pc * yslot + yo - ni);
      czp = ld4f(cs + oZP + pz * cslot + co);
    }
    {
      float xl = __shfl_up_sync(FULL, X0.w, 1), cxl = __shfl_up_sync(FULL, C.cx.w, 1);
      float xr = __shfl_down_sync(FULL, X0.x, 1);
      if (do_red && act_red) {
        if (warp_l && xlo) {
          xl = XZ ? 0.0f : cadd1(sm[x0 + xo - 1], px, j, i0 - 1);
          cxl = float(ldv(cs + oXP + pc * cslot + co - 1));
        }
        if (warp_r && need_r) xr = XZ ? 0.0f : cadd1(sm[x0 + xo + 4], px, j, i0 + 4);
        xl = xlo ? xl : 0.0f;
        xr = need_r ? xr : 0.0f;
        if (((j + p + 1) & 1) == 0) {
          X0.x = relax_quad_cell_m<0>(X0, xym, xyp, X1, xn, xl, xr, C, cxl, czp, pczp);
          X0.z = relax_quad_cell_m<2>(X0, xym, xyp, X1, xn, xl, xr, C, cxl, czp, pczp);
          if (PROLONG) {
            sm[x0 + xo] = X0.x;
            sm[x0 + xo + 2] = X0.z;
          }
        } else {
          X0.y = relax_quad_cell_m<1>(X0, xym, xyp, X1, xn, xl, xr, C, cxl, czp, pczp);
          X0.w = relax_quad_cell_m<3>(X0, xym, xyp, X1, xn, xl, xr, C, cxl, czp, pczp);
          if (PROLONG) {
            sm[x0 + xo + 1] = X0.y;
            sm[x0 + xo + 3] = X0.w;
          }
        }
        if (!PROLONG) *reinterpret_cast<float4*>(sm + x0 + xo) = X0;
      }
    }
    // No barrier here: the black pass of plane p-1 reads its own quad's red
    // update of plane p from registers and otherwise only values other
    // threads wrote in the previous step (rows j-1, j+1 of plane p-1 after
    // their red update); this step's red writes touch plane p only.

    // ---- black update of plane p-1 (tile rows) and the store
    const int q = p - 1;
    const bool do_blk = q >= k0 && q < kend;
    {
      float4 bym = z4, byp = z4;
      if (do_blk && act_blk) {
        if (ylo) bym = ld4f(sm + xm + xo - ni);
        if (yhi) byp = ld4f(sm + xm + xo + ni);
      }
      float xl = __shfl_up_sync(FULL, X1.w, 1), cxl = __shfl_up_sync(FULL, P.cx.w, 1);
      float xr = __shfl_down_sync(FULL, X1.x, 1);
      if (do_blk && act_blk) {
        if (warp_l && xlo) {
          xl = sm[xm + xo - 1];
          cxl = float(ldv(cs + oXP + scm1 * cslot + co - 1));
        }
        if (warp_r && need_r) xr = sm[xm + xo + 4];
        xl = xlo ? xl : 0.0f;
        xr = need_r ? xr : 0.0f;
        float4 o = X1;
        if (((j + q) & 1) == 0) {
          o.x = relax_quad_cell_m<0>(X1, bym, byp, X2, X0, xl, xr, P, cxl, pczp, pczm);
          o.z = relax_quad_cell_m<2>(X1, bym, byp, X2, X0, xl, xr, P, cxl, pczp, pczm);
        } else {
          o.y = relax_quad_cell_m<1>(X1, bym, byp, X2, X0, xl, xr, P, cxl, pczp, pczm);
          o.w = relax_quad_cell_m<3>(X1, bym, byp, X2, X0, xl, xr, P, cxl, pczp, pczm);
        }
        *reinterpret_cast<float4*>(a.x_out + (size_t)q * sz + (size_t)j * sy + i0) = o;
        if (DOT) dot += (double)o.x * P.bb.x + (double)o.y * P.bb.y + (double)o.z * P.bb.z + (double)o.w * P.bb.w;
      }
    }
    // rotate the carried state one plane on
    X2 = X1;
    X1 = X0;
    X0 = xn;
    pczm = pczp;
    pczp = czp;
    P = C;
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
