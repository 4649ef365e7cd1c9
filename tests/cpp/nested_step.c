/* SmokeSolver3D::time_step's FLIP step with its nested subdomain
 * (Smoke_solver3D.cpp:324-411) written against the C ABI, in the reference's
 * order.  Compiled as C by the tests to keep this integration sequence and
 * include/vflip.h in agreement; the scene code that
 * fills the buffers is the caller's.  All pointers are device memory, except
 * the counts written through the HOST int pointers. */
#include <stddef.h>

#include "vflip.h"

typedef struct {
  int ni, nj, nk;
  float h;
  const float* phi; /* nodal solid phi, (ni+1)(nj+1)(nk+1) */
  const int8_t* bdesc;
  const float *us, *vs, *ws; /* solid face velocities */
  float *u, *v, *w;          /* face velocities (updated) */
  float *uc, *vc, *wc, *du, *dv, *dw, *u0, *v0, *w0; /* P2G weights, deltas, pre-projection copies */
  double* pressure;
} grid_t;

/* One coupled step.  `flip` holds np main particles followed by the
 * subdomain's snp (appended by the caller: FLIP.push_back(sub_domain.FLIP)).
 * Returns 0 or the first failing status. */
int nested_flip_step(vflip_ctx* ctx, grid_t* g, grid_t* s, vflip_subdomain* sub, void* flip, int np, void* flip2,
                     int cap2, int* np_out, void* sflip, int scap, void* sflip2, int scap2, int* snp_out,
                     float* tracers, int nt, float* tracers2, int tcap, int* nt_out, float dt, unsigned seed) {
  int rc, snp = 0;
  vflip_solve_stats st, sst;
  const float L = (float)g->ni * g->h;
  const size_t nu = (size_t)(g->ni + 1) * g->nj * g->nk, nv = (size_t)g->ni * (g->nj + 1) * g->nk,
               nw = (size_t)g->ni * g->nj * (g->nk + 1);
  const size_t snu = (size_t)(s->ni + 1) * s->nj * s->nk, snv = (size_t)s->ni * (s->nj + 1) * s->nk,
               snw = (size_t)s->ni * s->nj * (s->nk + 1);
  /* emit_tracers / advect_tracers */
  if ((rc = vflip_emit_tracers_nested(ctx, tracers, nt, g->h, L, L, L, 0.5f * L, 0.1f * L, 0.5f * L, 0.1f * L, 1000,
                                      seed, g->ni, g->nj, g->nk, g->phi, sub, tracers2, tcap, nt_out)))
    return rc;
  if ((rc = vflip_advect_tracers_nested(ctx, g->ni, g->nj, g->nk, g->h, tracers2, *nt_out, g->u, g->v, g->w, g->phi,
                                        dt, 0.0f, sub)))
    return rc;
  /* advect_FLIP, hash_FLIP + particle_to_grid x3, pcg_projection, delta, particle_from_grid */
  if ((rc = vflip_advect_flip_nested(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->u, g->v, g->w, g->phi, dt, sub)))
    return rc;
  if ((rc = vflip_p2g(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->u, g->uc, g->v, g->vc, g->w, g->wc))) return rc;
  /* (the caller copies u, v, w to u0, v0, w0 here) */
  rc = vflip_project(ctx, g->ni, g->nj, g->nk, g->h, 0.0f, g->phi, g->bdesc, g->us, g->vs, g->ws, g->u, g->v, g->w,
                     g->pressure, 1e-6, 50, &st);
  if (rc < 0) return rc;
  if ((rc = vflip_delta(ctx, nu, g->u, g->u0, g->du)) || (rc = vflip_delta(ctx, nv, g->v, g->v0, g->dv)) ||
      (rc = vflip_delta(ctx, nw, g->w, g->w0, g->dw)))
    return rc;
  if ((rc = vflip_g2p(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->du, g->dv, g->dw, NULL, NULL, NULL, 1.0)))
    return rc;
  /* sub_domain.FLIP = the halo particles; its own pass */
  if ((rc = vflip_halo_select(ctx, flip, np, g->h, sub, sflip, scap, &snp))) return rc;
  if ((rc = vflip_sub_p2g(ctx, s->ni, s->nj, s->nk, s->h, sub->bmin[0], sub->bmin[1], sub->bmin[2], sflip, snp, s->u,
                          s->uc, s->v, s->vc, s->w, s->wc)))
    return rc;
  rc = vflip_project_subdomain(ctx, s->ni, s->nj, s->nk, s->h, 1.0f, s->phi, s->us, s->vs, s->ws, s->u, s->v, s->w,
                               s->pressure, 1e-9, 1000, &sst);
  if (rc < 0) return rc;
  if ((rc = vflip_delta(ctx, snu, s->u, s->u0, s->du)) || (rc = vflip_delta(ctx, snv, s->v, s->v0, s->dv)) ||
      (rc = vflip_delta(ctx, snw, s->w, s->w0, s->dw)))
    return rc;
  if ((rc = vflip_sub_g2p(ctx, s->ni, s->nj, s->nk, s->h, sub->bmin[0], sub->bmin[1], sub->bmin[2], sflip, snp, s->du,
                          s->dv, s->dw)))
    return rc;
  if ((rc = vflip_sub_reorder_flip(ctx, s->ni, s->nj, s->nk, s->h, sub->bmin[0], sub->bmin[1], sub->bmin[2], sflip,
                                   snp, s->u, s->v, s->w, s->phi, seed, sflip2, scap2, snp_out)))
    return rc;
  sub->u = s->u;
  sub->v = s->v;
  sub->w = s->w;
  /* reorder_FLIP with the nested solid filter */
  return vflip_reorder_flip_nested(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->u, g->v, g->w, g->phi, seed, flip2,
                                   cap2, np_out, sub);
}
