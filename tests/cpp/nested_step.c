/* SmokeSolver3D::time_step's FLIP step with its nested subdomain
 * (Smoke_solver3D.cpp:324-411) written against the C ABI, in the reference's
 * order.  The tests compile it as C99 against include/vflip.h and, on a GPU,
 * run it beside vflip_b200.flip.NestedFlipSim.step and require the same
 * particles and velocities byte for byte.  The scene code that fills the
 * buffers is the caller's.  All pointers are device memory, except the counts
 * written through the HOST int pointers. */
#include <stddef.h>

#include <cuda_runtime_api.h>

#include "vflip.h"

typedef struct {
  int ni, nj, nk;
  float h;
  const float* phi; /* nodal solid phi, (ni+1)(nj+1)(nk+1) */
  const int8_t* bdesc;
  const float *us, *vs, *ws; /* solid face velocities */
  float *u, *v, *w;          /* face velocities (written by P2G, updated by the projection) */
  float *uc, *vc, *wc, *du, *dv, *dw, *u0, *v0, *w0; /* P2G weights, deltas, pre-projection copies */
  double* pressure;
} grid_t;

/* The scene's emitter: called on the main grid's v faces after P2G, before
 * the pre-projection copy (the config-1 scene sets v on the faces inside its
 * source sphere to the inflow speed).  Returns 0 or a failing status. */
typedef int (*emitter_fn)(void* user, float* v);

typedef struct {
  float dt;
  double flip_ratio; /* 1.0: the reference's pure FLIP; <1 blends with the projected velocity (PIC) */
  unsigned seed;     /* the step's seed: the main reorder draws from it, the subdomain's from seed ^ 0x5EED */
  int tracer_count;  /* tracers emitted per step; 0 skips the tracer block */
  float src_c[3], src_r; /* tracer source sphere (world coordinates) */
  float dens_decay;      /* tracer density decay rate */
  emitter_fn emitter;    /* may be NULL */
  void* user;
  cudaStream_t stream;   /* the context's stream (vflip_config.stream) */
} step_params_t;

static int snapshot(cudaStream_t st, const grid_t* g) {
  const size_t nu = (size_t)(g->ni + 1) * g->nj * g->nk, nv = (size_t)g->ni * (g->nj + 1) * g->nk,
               nw = (size_t)g->ni * g->nj * (g->nk + 1);
  if (cudaMemcpyAsync(g->u0, g->u, nu * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(g->v0, g->v, nv * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(g->w0, g->w, nw * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return VFLIP_ERR_CUDA;
  return 0;
}

static int deltas(vflip_ctx* ctx, const grid_t* g) {
  const size_t nu = (size_t)(g->ni + 1) * g->nj * g->nk, nv = (size_t)g->ni * (g->nj + 1) * g->nk,
               nw = (size_t)g->ni * g->nj * (g->nk + 1);
  int rc;
  if ((rc = vflip_delta(ctx, nu, g->u, g->u0, g->du)) || (rc = vflip_delta(ctx, nv, g->v, g->v0, g->dv)) ||
      (rc = vflip_delta(ctx, nw, g->w, g->w0, g->dw)))
    return rc;
  return 0;
}

/* One coupled step.  `flip` holds np main particles followed by the
 * subdomain's (appended by the caller: FLIP.push_back(sub_domain.FLIP)), so np
 * counts both.  `tracers` (nt float4) may be NULL when tracer_count is 0.
 * Results: the reordered main particles in flip2 (*np_out), the subdomain's
 * in sflip2 (*snp_out), the tracers in tracers2 (*nt_out), the grids' new
 * velocities in g and s, and sub->u, v, w pointed at s's velocity.
 * Returns 0 or the first failing status. */
int nested_flip_step(vflip_ctx* ctx, const step_params_t* P, grid_t* g, grid_t* s, vflip_subdomain* sub, void* flip,
                     int np, void* flip2, int cap2, int* np_out, void* sflip, int scap, void* sflip2, int scap2,
                     int* snp_out, float* tracers, int nt, float* tracers2, int tcap, int* nt_out) {
  int rc, snp = 0;
  vflip_solve_stats st, sst;
  const float L = (float)g->ni * g->h;
  /* emit_tracers / advect_tracers */
  *nt_out = 0;
  if (P->tracer_count > 0) {
    if ((rc = vflip_emit_tracers_nested(ctx, tracers, nt, g->h, L, L, L, P->src_c[0], P->src_c[1], P->src_c[2],
                                        P->src_r, P->tracer_count, P->seed, g->ni, g->nj, g->nk, g->phi, sub,
                                        tracers2, tcap, nt_out)))
      return rc;
    if ((rc = vflip_advect_tracers_nested(ctx, g->ni, g->nj, g->nk, g->h, tracers2, *nt_out, g->u, g->v, g->w,
                                          g->phi, P->dt, P->dens_decay, sub)))
      return rc;
  }
  /* advect_FLIP, hash_FLIP + particle_to_grid x3 */
  if ((rc = vflip_advect_flip_nested(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->u, g->v, g->w, g->phi, P->dt,
                                     sub)))
    return rc;
  if ((rc = vflip_p2g(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->u, g->uc, g->v, g->vc, g->w, g->wc))) return rc;
  if (P->emitter && (rc = P->emitter(P->user, g->v))) return rc;
  /* _utemp.copy(_un) ... (Smoke_solver3D.cpp:374-376) */
  if ((rc = snapshot(P->stream, g))) return rc;
  /* pcg_projection, compute_delta_u, particle_from_grid */
  rc = vflip_project(ctx, g->ni, g->nj, g->nk, g->h, 0.0f, g->phi, g->bdesc, g->us, g->vs, g->ws, g->u, g->v, g->w,
                     g->pressure, 1e-6, 50, &st);
  if (rc < 0) return rc;
  if ((rc = deltas(ctx, g))) return rc;
  if ((rc = vflip_g2p(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->du, g->dv, g->dw, g->u, g->v, g->w,
                      P->flip_ratio)))
    return rc;
  /* sub_domain.FLIP = the halo particles; its own pass */
  if ((rc = vflip_halo_select(ctx, flip, np, g->h, sub, sflip, scap, &snp))) return rc;
  if ((rc = vflip_sub_p2g(ctx, s->ni, s->nj, s->nk, s->h, sub->bmin[0], sub->bmin[1], sub->bmin[2], sflip, snp, s->u,
                          s->uc, s->v, s->vc, s->w, s->wc)))
    return rc;
  /* the subdomain's compute_delta_u subtracts its own pre-projection copy */
  if ((rc = snapshot(P->stream, s))) return rc;
  rc = vflip_project_subdomain(ctx, s->ni, s->nj, s->nk, s->h, 1.0f, s->phi, s->us, s->vs, s->ws, s->u, s->v, s->w,
                               s->pressure, 1e-9, 1000, &sst);
  if (rc < 0) return rc;
  if ((rc = deltas(ctx, s))) return rc;
  if ((rc = vflip_sub_g2p(ctx, s->ni, s->nj, s->nk, s->h, sub->bmin[0], sub->bmin[1], sub->bmin[2], sflip, snp, s->du,
                          s->dv, s->dw)))
    return rc;
  /* the subdomain reseeds from its own stream of draws (seed ^ 0x5EED), so
   * main and subdomain reseeding never share random numbers */
  if ((rc = vflip_sub_reorder_flip(ctx, s->ni, s->nj, s->nk, s->h, sub->bmin[0], sub->bmin[1], sub->bmin[2], sflip,
                                   snp, s->u, s->v, s->w, s->phi, P->seed ^ 0x5EEDu, sflip2, scap2, snp_out)))
    return rc;
  sub->u = s->u;
  sub->v = s->v;
  sub->w = s->w;
  /* reorder_FLIP with the nested solid filter */
  return vflip_reorder_flip_nested(ctx, g->ni, g->nj, g->nk, g->h, flip, np, g->u, g->v, g->w, g->phi, P->seed, flip2,
                                   cap2, np_out, sub);
}
