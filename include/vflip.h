/* vflip.h - C ABI of the B200 (sm_100a) implementation of the vFLIP per-step
 * hot path: the MGPCG pressure projection, RK2 semi-Lagrangian advection and
 * the FLIP particle<->grid transfers.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns an int status (never aborts, never throws):
 *     VFLIP_OK (0)              success / solver converged
 *     VFLIP_NOT_CONVERGED (1)   solver hit max_iterations or met a zero/NaN
 *                               rho; the reference's `false`
 *     negative                  argument or CUDA error; vflip_last_error()
 *                               describes it.
 *
 * Memory: unless a parameter is documented as a host pointer, pointers are
 * device pointers on the context's device, and the call is ordered on the
 * context's stream (vflip_config.stream; NULL is the CUDA default stream).
 * Entry points that return solver statistics synchronise that stream.
 *
 * Grids are dense and linear, index = i + ni*(j + nj*k) (i fastest), the
 * order of the reference's pressure vector (Smoke_solver3D.cpp:993).  For an
 * ni x nj x nk cell grid of spacing h:
 *     cell   ni*nj*nk                 u faces (ni+1)*nj*nk
 *     v      ni*(nj+1)*nk             w faces ni*nj*(nk+1)
 *     nodal solid phi (ni+1)*(nj+1)*(nk+1)
 * A 7-point operator is passed as four FP64 arrays (diag, xp, yp, zp): the
 * diagonal and the couplings to the +x, +y, +z neighbours; the operator is
 * symmetric, so the -x coupling of cell c is xp[c-1].
 *
 * Reference file:line citations are paths inside the vFLIP project
 * (Smoke_Solver/ abbreviated SS/).
 */
#ifndef VFLIP_H
#define VFLIP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VFLIP_OK 0
#define VFLIP_NOT_CONVERGED 1
#define VFLIP_ERR_ARG (-1)
#define VFLIP_ERR_CUDA (-2)
#define VFLIP_ERR_NOT_7POINT (-3)
#define VFLIP_ERR_NOT_SYMMETRIC (-4)
#define VFLIP_ERR_NOMEM (-5)
#define VFLIP_ERR_TOO_LARGE (-6)

/* Arithmetic of the multigrid-preconditioned CG.
 *   FP64  - everything in FP64; the V-cycle is bit-identical to the
 *           reference's (the "FP64 GPU oracle solve").
 *   FP32  - vectors, operator and V-cycle in FP32; PCG inner products,
 *           residual norm and alpha/beta in FP64.
 *   MIXED - FP32 fine level, BF16 storage of the coarse-level operators,
 *           FP32 coarse vectors, FP64 scalars. */
typedef enum { VFLIP_PREC_FP64 = 0, VFLIP_PREC_FP32 = 1, VFLIP_PREC_MIXED = 2 } vflip_precision;

typedef struct {
  int precision;             /* vflip_precision, default VFLIP_PREC_FP32 */
  int pre_sweeps;            /* RBGS sweeps before restriction, default 4 (SS/AlgebraicMultigrid.h:156) */
  int post_sweeps;           /* RBGS sweeps after prolongation, default 4 (SS/AlgebraicMultigrid.h:164) */
  int coarse_sweeps;         /* RBGS sweeps on the coarsest level; 0 (default) = automatic: 200 in FP64
                                (SS/AlgebraicMultigrid.h:160), 100 in FP32/MIXED */
  int coarsest_max_unknowns; /* coarsen while unknowns exceed this (max 4096); 0 (default) = automatic:
                                4096 in FP64 (SS/GeometricLevelGen.h:46, the reference's hierarchy); in
                                FP32/MIXED 64 (a 4^3 coarsest level) with the direct coarsest solve, 512
                                (8^3) with the sweeps */
  int device;                /* CUDA device ordinal, default 0 */
  void* stream;              /* cudaStream_t to order work on; NULL: the CUDA default stream */
  int sweep_kernel;          /* smoother kernel: 0 (default) = automatic: for FP32 levels whose row length
                                is a multiple of 4, the TMA-pipelined kernel (bulk plane copies) in its
                                register-carry form (one thread per quad of a row for the whole march;
                                rows of up to 256 cells) or its plain form, else the plain fused kernel;
                                1 = always the plain fused kernel; 2 = 3-D-tiled (TMA tensor boxes,
                                several CTAs per SM) for FP32 levels whose row length is a multiple of 4
                                (8 for BF16 operators), else as 0; 3 = as 0; 4 = the TMA-pipelined kernel
                                without the register carry, else as 0.  All give the same bits. */
  /* Tile shape of the TMA-pipelined smoother, 0 = automatic (tuning knobs;
   * vflip_b200/tune.py searches them): copy groups in flight (1..3), output
   * rows per tile, plane ranges per launch, resident CTAs per SM (1..2),
   * threads per CTA (512 or 576), planes prefetched into L2 beyond the
   * copies in flight (1..8; -1 = none). */
  int smoother_depth;
  int smoother_tile_rows;
  int smoother_plane_ranges;
  int smoother_ctas_per_sm;
  int smoother_threads;
  int smoother_prefetch;
  /* Coarsest-level solve: 0 (default) = automatic: red-black sweeps
   * (coarse_sweeps) in FP64 contexts, the reference's; in FP32/MIXED
   * contexts an FP64 banded Cholesky direct solve, its factor built on the
   * GPU with each hierarchy, when the coarsest level's band (ni*nj of that
   * level) is at most 160 wide; the sweeps run instead where the band is
   * wider or a pivot shows the level singular (no open boundary pins some
   * fluid region).  1 = always the sweeps; 2 = the direct solve where it
   * applies, in every precision. */
  int coarsest_solver;
  /* PCG direction/SpMV kernel: 0 (default) = automatic: for fine levels
   * whose rows are whole warps of quads (ni a multiple of 128, at most 1024)
   * a plane-marching kernel (each s = z + beta s formed once, neighbours from
   * registers and a shared-memory plane ring), else the column kernel;
   * 1 = always the column kernel.  Both give the same q and s bit for bit;
   * their s.q partial sums are grouped differently. */
  int spmv_kernel;
  /* PCG loop: 0 (default) = automatic: the loop runs on the device, a CUDA
   * graph (captured once per hierarchy layout and reused) whose conditional
   * while node repeats V-cycle, direction, SpMV and update until the
   * device-side stop test holds, with one read of the scalars per solve -
   * unless per-launch profiling is on; 1 = the host loop, which reads the
   * scalars after every iteration.  Same iterates; a solve that does not
   * converge on the device is repeated by the host loop, so the failure
   * results (zero-rho exit, max_iterations) are the host loop's. */
  int pcg_loop;
  /* PCG vectors of FP32/MIXED contexts: 0 (default) = FP64: x, r, the
   * search direction and A s in FP64 and the SpMV on the FP64 operator as
   * assembled, around the FP32 (or BF16-coarse) V-cycle, which reads r
   * rounded to FP32; the |r|_inf <= tol |rhs|_inf test then holds for the
   * FP64 system.  1 = the working precision (vectors and SpMV in FP32: the
   * solve converges on the FP32-rounded system, whose FP64 residual stalls
   * near 2e-5 |rhs|_inf on the 256^3 plume operator). */
  int pcg_vectors;
  /* VFLIP_BATCH_PERSISTENT work items: cells per (system, level, chunk)
   * item and about the cells of a sweep tile (0 = automatic, 4096) and
   * resident CTAs per SM of the persistent
   * kernel (0 = as many as fit).  vflip_b200/tune.py picks both per batch. */
  int batch_chunk;
  int batch_ctas_per_sm;
  /* Small end of the V-cycle in FP32/MIXED contexts: 0 (default) =
   * automatic: every level from the first coarse level of at most 4096
   * cells down to the coarsest runs in ONE launch of one CTA (the levels in
   * shared memory, colour passes separated by CTA barriers), where that
   * level is not itself the coarsest; 1 = one launch per sweep, restriction
   * and coarsest solve.  Same bits. */
  int coarse_tail;
  /* Levels of at most this many cells (FP32/MIXED) sweep as independent 3-D
   * tiles of 16 x 8 x 4 cells, each staged with a two-cell halo and relaxed
   * in two barriers (no plane march: small levels live in L2 and the march's
   * per-plane latency dominated them); 0 (default) = automatic: 262144
   * (64^3); -1 = never.  The fine level's last sweep (which also forms z.r)
   * always marches.  Same bits. */
  int tile_sweep_max_cells;
  /* P2G gather on the main grid: 0 (default) = automatic, as 2; 1 = every
   * node gathers from global memory; 2 = tiled: a CTA stages the particles
   * of an 8 x 8 x 8 tile of face nodes and its one-cell ring in shared
   * memory (in chunks where they do not fit at once), one CTA per SM, and
   * its threads gather from there, two nodes each; 3 = the same with
   * 8 x 8 x 4 tiles, two CTAs per SM.  Same bits. */
  int p2g_kernel;
  /* RK2 trilinear advection in FP32/MIXED contexts: 0 (default) =
   * automatic: when h is a power of two and the field lies on the u, v, w or
   * cell-centre lattice, the backtrace's first stage is read straight from
   * the node's neighbours (its axis fractions are exactly 0 or 1/2) and
   * u, v, w advect in one launch; otherwise as 1; 1 = every sample through
   * the general trilinear transform, one launch per field.  Same bits. */
  int advect_kernel;
} vflip_config;

typedef struct {
  int iterations;   /* PCG iterations (the reference's iterations_out) */
  int vcycles;      /* V-cycle applications, iterations + 1 when any ran */
  int levels;       /* multigrid levels */
  int converged;    /* 1 when |r|_inf <= tol * |rhs|_inf */
  double residual;  /* |r|_inf at exit (the reference's residual_out) */
  double rhs_norm;  /* |rhs|_inf */
  double solve_ms;  /* device time of the solve, hierarchy build included */
} vflip_solve_stats;

typedef struct vflip_ctx vflip_ctx;

/* Fills *cfg with the reference's defaults. */
void vflip_config_default(vflip_config* cfg);
/* sizeof(vflip_config) in this build of the library.  vflip_config grows by
 * fields appended at its end; code compiled against another version of this
 * header compares it with its own sizeof(vflip_config) and must not pass its
 * struct to the library when they differ. */
size_t vflip_config_size(void);

/* Creates a context (device buffers are allocated lazily and reused across
 * calls of the same size).  One context per host thread. */
int vflip_create(vflip_ctx** out, const vflip_config* cfg);
int vflip_destroy(vflip_ctx* ctx);
/* Text of the last error on this context ("" when none). */
const char* vflip_last_error(const vflip_ctx* ctx);
int vflip_synchronize(vflip_ctx* ctx);
/* Device time in milliseconds of the most recent solve or step. */
double vflip_last_ms(const vflip_ctx* ctx);

/* ---- MGPCG ------------------------------------------------------------- */

/* Drop-in for
 *   template<class T> bool ivock::AMGPCGSolve(const SparseMatrix<T>& matrix,
 *       const std::vector<T>& rhs, std::vector<T>& result, T tolerance_factor,
 *       int max_iterations, T& residual_out, int& iterations_out,
 *       int ni, int nj, int nk)                 (SS/AlgebraicMultigrid.h:189-197)
 * with the matrix as CSR (rows sorted by column, as FixedSparseMatrix holds
 * it, SS/sparse_matrix.h:266-312).  ALL POINTERS ARE HOST POINTERS.  The
 * matrix must be the 7-point, symmetric operator of an ni x nj x nk grid
 * (what pcg_projection assembles); otherwise VFLIP_ERR_NOT_7POINT /
 * VFLIP_ERR_NOT_SYMMETRIC.  result (n) is zeroed and written; the return
 * value is VFLIP_OK where the reference returns true, VFLIP_NOT_CONVERGED
 * where it returns false. */
int vflip_amgpcg_solve_csr(vflip_ctx* ctx, uint32_t n, const uint32_t* rowstart, const uint32_t* colindex,
                           const double* value, const double* rhs, double* result, double tolerance_factor,
                           int max_iterations, double* residual_out, int* iterations_out, int ni, int nj, int nk);

/* Same solve on a device-resident stencil operator and device vectors:
 * rhs and result are FP64 arrays of ni*nj*nk.  stats may be NULL. */
int vflip_amgpcg_solve(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp,
                       const double* yp, const double* zp, const double* rhs, double* result,
                       double tolerance_factor, int max_iterations, vflip_solve_stats* stats);

/* Galerkin hierarchy (SS/GeometricLevelGen.h:28-71, .cpp:7-76) of an FP64
 * stencil operator.  dims_out (HOST, 3*max_levels ints) receives each
 * level's size; levels_out (device, may be NULL) receives, level after
 * level, the four FP64 arrays diag, xp, yp, zp of each level.  Returns the
 * number of levels (>= 1) or a negative status. */
int vflip_build_levels(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp,
                       const double* yp, const double* zp, int max_levels, int* dims_out, double* levels_out);

/* `iterations` red-black Gauss-Seidel sweeps in place on x (FP64),
 * ivock::RBGS (SS/AlgebraicMultigrid.h:22-103). */
int vflip_rbgs(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp, const double* yp,
               const double* zp, const double* b, double* x, int iterations);

/* x = one V-cycle applied to b from x = 0, ivock::amgPrecond
 * (SS/AlgebraicMultigrid.h:130-188), in the context's precision (b and x
 * are FP64 either way). */
int vflip_vcycle(vflip_ctx* ctx, int ni, int nj, int nk, const double* diag, const double* xp, const double* yp,
                 const double* zp, const double* b, double* x);

/* Same sweeps as vflip_rbgs, for callers that cannot allocate device memory:
 * code recorded into a CUDA graph by stream capture (where cudaMalloc is not
 * permitted), real-time loops that forbid allocation, and applications that
 * hand every device byte to their own allocator.  No context is needed and
 * nothing is allocated: the work runs on `stream` (NULL: the default stream)
 * of the current device, and the second buffer of the sweeps is a fixed
 * array of VFLIP_NOALLOC_MAX_CELLS doubles (2 MiB) inside this library, which
 * every GPU that loads the library holds until the process exits.  Grids with
 * more than VFLIP_NOALLOC_MAX_CELLS cells return VFLIP_ERR_TOO_LARGE.
 * The first call on a device looks up that array's device address (once per
 * device) and must come before any stream capture on that device.  All calls
 * share the one array: calls that overlap on the GPU (different streams, or
 * different host threads) race on it and must be serialised by the caller.
 * The array keeps the last call's contents; every sweep overwrites all the
 * cells it reads back, so nothing needs clearing.  No counterpart in the
 * reference (its RBGS, AlgebraicMultigrid.h:22-103, allocates host vectors). */
#define VFLIP_NOALLOC_MAX_CELLS (64 * 64 * 64)
int vflip_rbgs_noalloc(void* stream, int ni, int nj, int nk, const double* diag, const double* xp, const double* yp,
                       const double* zp, const double* b, double* x, int iterations);

/* ---- pressure projection -------------------------------------------------- */

/* Face open fractions from the nodal solid level set,
 * SmokeSolver3D::compute_face_weights (SS/Smoke_solver3D.cpp:874-944). */
int vflip_face_weights(vflip_ctx* ctx, int ni, int nj, int nk, const float* nodal_phi, float* uw, float* vw,
                       float* ww);

/* Assembles the projection's operator and rhs without solving
 * (SS/Smoke_solver3D.cpp:964-1111, inflow overwrite applied to u/v/w in
 * place).  diag/xp/yp/zp/rhs are FP64 cell arrays. */
int vflip_assemble(vflip_ctx* ctx, int ni, int nj, int nk, float h, float U_in, const float* nodal_phi,
                   const int8_t* bdesc, const float* us, const float* vs, const float* ws, float* u, float* v,
                   float* w, double* diag, double* xp, double* yp, double* zp, double* rhs);

/* SmokeSolver3D::pcg_projection (SS/Smoke_solver3D.cpp:945-1202): face
 * weights, inflow overwrite, assembly, MGPCG to tolerance_factor (the
 * reference uses 1e-6, 50 iterations), gradient update of u/v/w in place.
 * pressure (FP64 cells) may be NULL; stats may be NULL.  Returns the solve's
 * status. */
int vflip_project(vflip_ctx* ctx, int ni, int nj, int nk, float h, float U_in, const float* nodal_phi,
                  const int8_t* bdesc, const float* us, const float* vs, const float* ws, float* u, float* v,
                  float* w, double* pressure, double tolerance_factor, int max_iterations,
                  vflip_solve_stats* stats);

/* SubDomainSolver::pcg_projection (SS/sub_domain.cpp:560-821), the nested
 * fine domain's projection: no inflow overwrite, operator terms
 * w*dt/h^2, solid term scaled by the float 1/h, and the gradient
 * u -= dt*(p_i - p_{i-1})/h applied on every face between two cells of the
 * grid.  The reference solves it to tolerance 1e-9 in at most 1000
 * iterations (SS/sub_domain.cpp:739). */
int vflip_project_subdomain(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* nodal_phi,
                            const float* us, const float* vs, const float* ws, float* u, float* v, float* w,
                            double* pressure, double tolerance_factor, int max_iterations,
                            vflip_solve_stats* stats);

/* ---- advection ------------------------------------------------------------- */

/* Semi-Lagrangian RK2 (midpoint) backtrace through the MAC velocity u/v/w of
 * an ni x nj x nk grid of spacing h, then a trilinear sample of `field`,
 * SubDomainSolver::advect_field (SS/sub_domain.cpp:191-235).  field/out are
 * fnx x fny x fnz grids of spacing h whose node (i,j,k) sits at world
 * ((i-ox)h, (j-oy)h, (k-oz)h): (0.5,0,0) for u, (0,0.5,0) for v, (0,0,0.5)
 * for w, (0,0,0) for cell-centred scalars.  out must not alias field or u/v/w.
 * A VFLIP_PREC_FP64 context reproduces the reference's FP64 sampling bit for
 * bit; FP32/MIXED contexts sample in FP32 (a few ulp from it). */
int vflip_advect_rk2_linear(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                            const float* v, const float* w, int fnx, int fny, int fnz, double ox, double oy,
                            double oz, const float* field, float* out);

/* Same backtrace for two fields on one grid (e.g. density and temperature):
 * out = advect(field), out2 = advect(field2); field2/out2 may be NULL. */
int vflip_advect_rk2_linear2(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                             const float* v, const float* w, int fnx, int fny, int fnz, double ox, double oy,
                             double oz, const float* field, float* out, const float* field2, float* out2);

/* The velocity's self-advection of SubDomainSolver::advect_field
 * (SS/sub_domain.cpp:191-235) for u, v and w in one call: uo, vo, wo (the
 * face grids, which must not alias u/v/w) receive what three
 * vflip_advect_rk2_linear calls give (it makes those three launches). */
int vflip_advect_velocity_rk2_linear(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                                     const float* v, const float* w, float* uo, float* vo, float* wo);

/* SmokeSolver3D::advect_field_cubic_clamp (SS/Smoke_solver3D.cpp:657-707):
 * the RK2 backtrace above, then the cubic sample of Buffer3D::sample_cubic
 * (SS/fluid_buffer3D.h:22-38, 259-326) over the clamped 4x4x4 neighbourhood,
 * replaced by the trilinear sample where the cubic value reaches or leaves
 * the range of the eight surrounding nodes.  Arguments as
 * vflip_advect_rk2_linear; FP64 contexts are bit-identical to the reference,
 * FP32/MIXED contexts run the same scheme in FP32. */
int vflip_advect_cubic_clamp(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                             const float* v, const float* w, int fnx, int fny, int fnz, double ox, double oy,
                             double oz, const float* field, float* out);

/* SmokeSolver3D::advect (SS/Smoke_solver3D.cpp:8-29): cubic-clamped
 * self-advection of the MAC velocity, all three components in one launch.
 * The outputs must not alias the inputs. */
int vflip_advect_velocity_cubic_clamp(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                                      const float* v, const float* w, float* u_out, float* v_out, float* w_out);

/* SmokeSolver3D::advect_field (SS/Smoke_solver3D.cpp:564-610): traceRK3
 * (SS/Smoke_solver3D.cpp:144-157) from each node with step -dt through the
 * MAC velocity of the ni x nj x nk grid of spacing h, then a trilinear
 * sample.  The field has its own spacing fh: node (i,j,k) sits at
 * ((i-ox)fh, (j-oy)fh, (k-oz)fh).  The reference's density and temperature
 * grids are 2ni x 2nj x 2nk at fh = h/2 with zero offsets
 * (SS/Smoke_solver3D.h:313-315).  Precision as vflip_advect_cubic_clamp. */
int vflip_advect_rk3_linear(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                            const float* v, const float* w, int fnx, int fny, int fnz, double fh, double ox,
                            double oy, double oz, const float* field, float* out);

/* Same for two fields on one grid sharing the backtrace (density and
 * temperature); field2/out2 may be NULL. */
int vflip_advect_rk3_linear2(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, const float* u,
                             const float* v, const float* w, int fnx, int fny, int fnz, double fh, double ox,
                             double oy, double oz, const float* field, float* out, const float* field2,
                             float* out2);

/* ---- smoke scalars on the density/temperature grids ------------------------ */

/* SmokeSolver3D::gen_heat (SS/Smoke_solver3D.cpp:1624-1650), in place on the
 * fnx x fny x fnz density and temperature grids of spacing fh: divide by
 * (1 + decay dt), then set (dens, heat) inside the source, the nodes
 * (i,j,k) fh within `radius` of (cx, cz) horizontally and within radius/4 of
 * cy vertically.  Bit-identical to the reference. */
int vflip_gen_heat(vflip_ctx* ctx, int fnx, int fny, int fnz, double fh, float dt, float dens_decay,
                   float temp_decay, float cx, float cy, float cz, float radius, float dens, float heat, float* rho,
                   float* temp);

/* SmokeSolver3D::add_smokeforce (SS/Smoke_solver3D.cpp:1652-1668): each
 * particle's y velocity gains dt (-alpha rho + beta T), with rho and T
 * sampled trilinearly (FP64 lerps) from the grids of spacing fh.  In place;
 * bit-identical to the reference. */
int vflip_add_smokeforce(vflip_ctx* ctx, void* particles, int np, int fnx, int fny, int fnz, double fh,
                         const float* rho, const float* temp, float alpha, float beta, float dt);

/* ---- nested subdomain particle transfers ----------------------------------
 * A SubDomainSolver grid (SS/sub_domain.h, SS/sub_domain.cpp): ni x nj x nk
 * cells of spacing h whose origin sits at bmin = (bx, by, bz) in world space;
 * particles keep world positions and every sample is taken at pos - bmin
 * (float).  Face grids have the main grid's shapes and offsets.  All four
 * are bit-identical to the reference's (new particles: counter-based draws,
 * as vflip_reorder_flip). */

/* SubDomainSolver::hash_FLIP (SS/sub_domain.cpp:1087-1109): the cell of
 * pos - bmin + h/2, truncated and clamped into the grid (every particle has
 * a cell). */
int vflip_sub_particle_cells(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz,
                             const void* particles, int np, int* cell_out);

/* SubDomainSolver::particle_to_grid (SS/sub_domain.cpp:1204-1265) after
 * hash_FLIP, for the components whose pointers are given: within 4 cells of
 * the subdomain's boundary the tent is 4h wide over the 9^3 neighbouring
 * cells (determineDist, SS/sub_domain.h:89-103), elsewhere h over 3^3. */
int vflip_sub_p2g(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz,
                  const void* particles, int np, float* u, float* ucoef, float* v, float* vcoef, float* w,
                  float* wcoef);

/* SubDomainSolver::particle_from_grid (SS/sub_domain.cpp:1161-1178): vel +=
 * the delta grids sampled at pos - bmin, in place. */
int vflip_sub_g2p(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz, void* particles,
                  int np, const float* du, const float* dv, const float* dw);

/* SubDomainSolver::hash_FLIP + reorder_FLIP (SS/sub_domain.cpp:1087-1159): as
 * vflip_reorder_flip over the interior cells (1 .. n-2 on each axis) only,
 * new particles at bmin + (i,j,k) h + r 0.49 h with the subdomain's velocity,
 * filtered on the subdomain's nodal solid phi. */
int vflip_sub_reorder_flip(vflip_ctx* ctx, int ni, int nj, int nk, float h, float bx, float by, float bz,
                           const void* particles, int np, const float* u, const float* v, const float* w,
                           const float* nodal_phi, unsigned seed, void* out, int capacity, int* np_out);

/* ---- the main grid with its nested subdomain active --------------------------
 *
 * SmokeSolver3D's samplers defer to its SubDomainSolver inside the
 * subdomain's box (SS/Smoke_solver3D.cpp:61-124, SS/sub_domain.cpp:61-105):
 *   get_velocity    inside is_in2 (5 h_s from the box faces) the main grid's
 *                   velocity v becomes c v_sub + (1 - c) v, v_sub sampled at
 *                   pos - bmin, c = get_boundary_coef (the distance to the box
 *                   5 h_s inside, over 4 h_s, clamped to [0, 1]);
 *   get_solid_phi / get_solid_normal
 *                   inside is_in (2 h_s) the subdomain's nodal phi at
 *                   pos - bmin (its gradient with spacing h_s).
 * The calls below are the main solver's routines with those samplers; the
 * subdomain's own routines are the vflip_sub_* calls above. */

/* A nested subdomain: ni x nj x nk cells of spacing h at bmin (bmax =
 * bmin + (ni, nj, nk) h), its face velocities and nodal solid phi (device,
 * linear layout). */
typedef struct vflip_subdomain {
  int ni, nj, nk;
  float h;
  float bmin[3];
  const float* u;
  const float* v;
  const float* w;
  const float* nodal_phi;
} vflip_subdomain;

/* vflip_advect_flip through the nested samplers (advect_FLIP,
 * SS/Smoke_solver3D.cpp:1407-1449, with the subdomain active). */
int vflip_advect_flip_nested(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np,
                             const float* u, const float* v, const float* w, const float* nodal_phi, float dt,
                             const vflip_subdomain* sub);

/* vflip_reorder_flip whose final solid filter is the nested get_solid_phi
 * (reorder_FLIP, SS/Smoke_solver3D.cpp:1347-1396, with the subdomain active;
 * new particles still take the main grid's velocity). */
int vflip_reorder_flip_nested(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                              const float* u, const float* v, const float* w, const float* nodal_phi, unsigned seed,
                              void* out, int capacity, int* np_out, const vflip_subdomain* sub);

/* The halo selection of SmokeSolver3D::time_step (SS/Smoke_solver3D.cpp:390-398):
 * copies, in order, the particles strictly inside [bmin - dx, bmax + dx] on
 * every axis (SubDomainSolver::is_halo, SS/sub_domain.h:202-213) with
 * dx = 0.5 h, h the MAIN grid's spacing, to `out` (device, `capacity`
 * records); *n_out (HOST) gets the count (VFLIP_ERR_TOO_LARGE when it
 * exceeds capacity).  Synchronises the stream. */
int vflip_halo_select(vflip_ctx* ctx, const void* particles, int np, float h, const vflip_subdomain* sub, void* out,
                      int capacity, int* n_out);

/* vflip_advect_tracers through the nested samplers (advect_tracers,
 * SS/Smoke_solver3D.h:99-120, with the subdomain active). */
int vflip_advect_tracers_nested(vflip_ctx* ctx, int ni, int nj, int nk, float h, float* tracers, int n,
                                const float* u, const float* v, const float* w, const float* nodal_phi, float dt,
                                float dens_decay, const vflip_subdomain* sub);

/* emit_tracers with the subdomain's seeding (SS/Smoke_solver3D.h:46-96):
 * vflip_emit_tracers, then for each subdomain cell in (k, j, i) order four
 * candidates at bmin + (i, j, k) h_s + r h_s (r uniform in [0, 1)^3) of
 * density 1, kept where the nested solid phi over the main grid's nodal_phi
 * (ni x nj x nk cells of spacing h) lies in (0, h_s).  The reference draws r
 * from rand(); here r comes from a counter-based hash of (seed, cell, slot,
 * axis).  *n_out gets the total; VFLIP_ERR_TOO_LARGE when it exceeds
 * `capacity`.  Synchronises the stream. */
int vflip_emit_tracers_nested(vflip_ctx* ctx, const float* tracers, int n, float h, float lx, float ly, float lz,
                              float cx, float cy, float cz, float r, int count, unsigned seed, int ni, int nj, int nk,
                              const float* nodal_phi, const vflip_subdomain* sub, float* out, int capacity,
                              int* n_out);

/* ---- smoke tracers (float4 records: x, y, z, density) ----------------------- */

/* SmokeSolver3D::emit_tracers (SS/Smoke_solver3D.h:46-85): keeps, in order,
 * the tracers inside [2h, L-2h] on every axis (L = lx, ly, lz) whose density
 * exceeds 0.01, then appends `count` new ones of density 1 uniform in the
 * sphere of radius r about (cx, cy, cz).  The reference rejection-samples
 * rand() over a cube of half-width r + h; this library rejection-samples a
 * counter-based hash of (seed, slot, attempt) over the sphere's bounding
 * cube: the same law, other positions.  The nested subdomain's seeding
 * (:86-96) is vflip_emit_tracers_nested.  `out` (capacity float4, must not alias
 * `tracers`) receives the result and *n_out (HOST) its count; when that
 * exceeds `capacity` nothing is written and VFLIP_ERR_TOO_LARGE returns.
 * Synchronises the stream. */
int vflip_emit_tracers(vflip_ctx* ctx, const float* tracers, int n, float h, float lx, float ly, float lz, float cx,
                       float cy, float cz, float r, int count, unsigned seed, float* out, int capacity, int* n_out);

/* SmokeSolver3D::advect_tracers (SS/Smoke_solver3D.h:99-120), in place:
 * traceRK3 through the MAC velocity, out of a solid along its normal where
 * the sampled nodal phi is <= 0, density / (1 + dens_decay dt).
 * Bit-identical to the reference. */
int vflip_advect_tracers(vflip_ctx* ctx, int ni, int nj, int nk, float h, float* tracers, int n, const float* u,
                         const float* v, const float* w, const float* nodal_phi, float dt, float dens_decay);

/* SmokeSolver3D::write_tracers (SS/Smoke_solver3D.h:121-160): writes
 * <dir>/Particle_data%04d.bin (frame) holding n float4 records
 * (x/lx - 0.5, y/lx, z/lx - 0.5, density), the reference's byte layout.
 * `dir` is a HOST string; synchronises the stream. */
int vflip_write_tracers(vflip_ctx* ctx, const float* tracers, int n, float lx, const char* dir, int frame);

/* delta = after - before, n floats (SmokeSolver3D::getDelta, SS/Smoke_solver3D.cpp:1298-1319). */
int vflip_delta(vflip_ctx* ctx, size_t n, const float* after, const float* before, float* delta);

/* ---- FLIP transfers (particles: the reference's 40-byte `particle` records,
 *      SS/fluid_particle.h:14-20: pos f32x3, vel f32x3, dens, temp,
 *      hash_idx, sub_hash_idx) ------------------------------------------------ */

/* Cell of each particle as SmokeSolver3D::hash_FLIP computes it
 * (SS/Smoke_solver3D.cpp:1327-1346); -1 when outside the grid. */
int vflip_particle_cells(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                         int* cell_out);

/* SmokeSolver3D::particle_to_grid for u, v and w (SS/Smoke_solver3D.cpp:
 * 1451-1510) after hash_FLIP: field = sum(w*vel)/sum(w), coef = sum(w) on
 * each face grid, summed in the reference's bucket order (sort by cell,
 * deterministic).  Any output pair may be NULL to skip that component. */
int vflip_p2g(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np, float* u,
              float* ucoef, float* v, float* vcoef, float* w, float* wcoef);

/* SmokeSolver3D::particle_from_grid (SS/Smoke_solver3D.cpp:1398-1406):
 * vel += trilinear(du, dv, dw) when flip_ratio == 1; otherwise
 * vel = (1-flip_ratio) u_new(pos) + flip_ratio (vel + delta(pos)), the blend
 * of fluid_particle::interpolate (SS/fluid_particle.h:315-328).  un/vn/wn
 * may be NULL when flip_ratio == 1.  particles are updated in place. */
int vflip_g2p(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np, const float* du,
              const float* dv, const float* dw, const float* un, const float* vn, const float* wn,
              double flip_ratio);

/* SmokeSolver3D::advect_FLIP (SS/Smoke_solver3D.cpp:1407-1449): RK3 trace
 * through the grid velocity (traceRK3 :144-158, with the reference's
 * c3 = (1 - c1 - c2) dt), then a particle whose sampled nodal solid phi is
 * negative moves out along the normalised phi gradient by -phi
 * (get_solid_normal :115-124).  Positions updated in place; bit-exact. */
int vflip_advect_flip(vflip_ctx* ctx, int ni, int nj, int nk, float h, void* particles, int np, const float* u,
                      const float* v, const float* w, const float* nodal_phi, float dt);

/* SmokeSolver3D::hash_FLIP + reorder_FLIP (SS/Smoke_solver3D.cpp:1327-1396):
 * per cell in (k, j, i) order, fewer than 8 particles are kept and topped up
 * to 8 with new ones at (i, j, k) h + r 0.49 h (r uniform in [-1, 1)^3, grid
 * velocity there, density/temperature 0), 8-9 kept, 10+ cut to their first
 * 8; then particles inside solids (sampled nodal phi < 0) are dropped.  The
 * reference draws r from rand(); here r comes from a counter-based hash of
 * (seed, cell, slot, axis), so new positions differ from the reference's
 * while the kept particles, their order and the counts match.  Writes the
 * result to `out` (device, `capacity` records) and its count to *np_out
 * (also when it exceeds capacity: VFLIP_ERR_TOO_LARGE). */
int vflip_reorder_flip(vflip_ctx* ctx, int ni, int nj, int nk, float h, const void* particles, int np,
                       const float* u, const float* v, const float* w, const float* nodal_phi, unsigned seed,
                       void* out, int capacity, int* np_out);

/* ---- measurement ----------------------------------------------------------- */

/* When enabled, every launch of the kinds below is bracketed by a pair of
 * CUDA events on its stream (the PCG loop then runs on the host, whose
 * launches can carry events): the fine-level smoothing sweep (the dominant
 * kernel), the fine-level PCG SpMV and update, and the RK2 advection
 * launches (one field; a pair of fields on one backtrace); and, as spans of
 * several launches, each V-cycle of the PCG (VCYCLE) and its part below the
 * fine level (COARSE: the levels >= 1, from after the fine restriction to
 * the fine prolongation); P2G_SORT spans a P2G's bucketing (histogram,
 * scan, scatter, bucket sort, sorted copies), P2G_GATHER its gathers.
 * vflip_profile_kernels synchronises the stream and returns the
 * number of timed launches of one kind and their summed device time;
 * vflip_profile_sweeps returns the fine sweeps' figures and the fine level's
 * cell count, then starts a new count for every kind.  Enabling (again)
 * also starts a new count.  No reference counterpart. */
#define VFLIP_PROF_FINE_SWEEP 0
#define VFLIP_PROF_SPMV 1
#define VFLIP_PROF_UPDATE 2
#define VFLIP_PROF_ADVECT_FIELD 3
#define VFLIP_PROF_ADVECT_PAIR 4
#define VFLIP_PROF_VCYCLE 5
#define VFLIP_PROF_COARSE 6
#define VFLIP_PROF_P2G_SORT 7
#define VFLIP_PROF_P2G_GATHER 8
int vflip_set_profiling(vflip_ctx* ctx, int enable);
int vflip_profile_sweeps(vflip_ctx* ctx, int* launches, double* total_ms, double* cells);
int vflip_profile_kernels(vflip_ctx* ctx, int kind, int* launches, double* total_ms);
/* Number of kernels launched through this context so far. */
unsigned long long vflip_launch_count(const vflip_ctx* ctx);

/* ---- plume scenes ---------------------------------------------------------- */

/* Grid analogue of the reference's smoke sources (SS/Smoke_solver3D.cpp:
 * 1624-1668, which act on particles and 2x density/temperature grids): sets
 * rho = dens_value and temp = heat_value in the cells whose centre (i,j,k)*h
 * lies in the sphere (cx,cy,cz, radius), then adds
 * dt * (-alpha * rho + beta * temp), averaged over the two adjacent cells, to
 * every interior v face.  No reference counterpart on the grid path. */
int vflip_plume_sources(vflip_ctx* ctx, int ni, int nj, int nk, float h, float dt, float* rho, float* temp, float* v,
                        float cx, float cy, float cz, float radius, float dens_value, float heat_value, float alpha,
                        float beta);

/* ---- layout --------------------------------------------------------------- */

/* Buffer3D's 8^3-bricked storage (SS/fluid_buffer3D.h:86-104, 186-202) <->
 * this library's linear layout, for an nx x ny x nz float grid.  The bricked
 * array holds ceil(n/8)*8 elements per axis. */
int vflip_bricks_to_linear(vflip_ctx* ctx, int nx, int ny, int nz, const float* bricked, float* linear);
int vflip_linear_to_bricks(vflip_ctx* ctx, int nx, int ny, int nz, const float* linear, float* bricked);

/* ---- learned preconditioner: the 3D U-Net --------------------------------- */

/* No reference counterpart (the reference solves with plain MGPCG only).  A
 * 3D U-Net (4 levels, 16/32/64/128 channels, 3x3x3 convolutions with ReLU,
 * 2x2x2 average pooling, nearest upsampling, concatenated skips) maps
 * (scaled rhs, fluid fraction) on a coarse grid to two fields: a warm-start
 * pressure and a coarse correction.  Convolutions are BF16 tensor-core
 * (tcgen05) kernels with FP32 accumulation; parameters are FP32 masters,
 * trained by Adam with the library's own backward kernels.  All array
 * arguments are device pointers ordered on `stream` (NULL = the default
 * stream).  Network grids have dimensions that are multiples of 8; per-voxel
 * fields are channels-last [z][y][x][c]. */
typedef struct vflip_unet vflip_unet;
int vflip_unet_create(vflip_unet** net, int device, void* stream, unsigned long long seed);
int vflip_unet_destroy(vflip_unet* net);
const char* vflip_unet_last_error(const vflip_unet* net);
/* number of FP32 parameters: per layer W[cout][cin][27] then b[cout] */
int vflip_unet_num_params(void);
int vflip_unet_get_params(vflip_unet* net, float* host_params);
int vflip_unet_set_params(vflip_unet* net, const float* host_params); /* also resets Adam */
/* in2, out2: [Z][Y][X][2] FP32 */
int vflip_unet_forward(vflip_unet* net, int X, int Y, int Z, const float* in2, float* out2);
/* loss = sum_v weight[v] (cw0 (o0 - t0)^2 + cw1 (o1 - t1)^2) / (X Y Z); grad_out: nparams FP32 (or NULL) */
int vflip_unet_gradients(vflip_unet* net, int X, int Y, int Z, const float* in2, const float* target2,
                         const float* weight, float cw0, float cw1, float* grad_out, double* loss);
/* one Adam step (beta 0.9 / 0.999) on that loss */
int vflip_unet_train_step(vflip_unet* net, int X, int Y, int Z, const float* in2, const float* target2,
                          const float* weight, float cw0, float cw1, float lr, double* loss);
/* Single 3x3x3 convolution (zero padding) of a BF16 channel view
 * in[v*in_ctot + in_coff + c] with FP32 weights w[layer_cout][layer_cin][27]
 * (tap = 9 dz + 3 dy + dx, offsets -1..1).  backward_data = 0: out = conv(in)
 * + bias, ReLU if relu; backward_data = 1: the gradient with respect to the
 * layer's input (layer_cout channels in, layer_cin out, taps mirrored, no
 * bias).  mask (optional) zeroes outputs where mask <= 0.  Output as BF16
 * (out) and/or FP32 (outf, first outf_valid channels). */
int vflip_unet_conv3(vflip_unet* net, int X, int Y, int Z, const void* in, int in_ctot, int in_coff, const float* w,
                     int layer_cin, int layer_cout, int backward_data, const float* bias, int relu, const void* mask,
                     int mask_ctot, int mask_coff, void* out, int out_ctot, int out_coff, float* outf, int outf_stride,
                     int outf_valid);
/* dw[cout][cin][27] = sum_v dy[v][co] * x[v + tap][ci] (FP32, deterministic) */
int vflip_unet_conv3_wgrad(vflip_unet* net, int X, int Y, int Z, const void* x, int x_ctot, int x_coff, int cin,
                           const void* dy, int dy_ctot, int dy_coff, int cout, float* dw);
long long vflip_unet_launch_count(const vflip_unet* net);
/* Multipliers of the two outputs when a learned solve uses them (training
 * sets them to the RMS its targets were divided by); default 1. */
int vflip_unet_set_output_scale(vflip_unet* net, float s0, float s1);

/* ---- learned-preconditioned projection -------------------------------------- */

/* mode bits of vflip_project_learned */
#define VFLIP_LEARNED_CAPTURE 1 /* plain MGPCG; also write this solve's training triple */
#define VFLIP_LEARNED_SOLVE 2   /* network warm start + coarse correction, flexible PCG */
#define VFLIP_LEARNED_NO_VB 4   /* leave V(b) out of the initial Ritz subspace */
#define VFLIP_LEARNED_PREV 8    /* add the incoming pressure (previous solve) to the Ritz subspace */
#define VFLIP_LEARNED_NO_NET 16 /* leave the network out (ablation; net may be NULL) */
#define VFLIP_LEARNED_SWEEPS(k) ((k) << 8) /* k (0-15) smoothing sweeps on each network vector */
#define VFLIP_LEARNED_RESID 32  /* warm-start correction: the network maps the residual r0 = b - A p of the
                                   previous pressure p (the pressure array on entry) to a correction of p; capture
                                   records (r0 features, R^L(p_new - p)); solve takes the energy-optimal
                                   combination of p and the smoothed correction (p alone with NO_NET), then PCG
                                   with the plain V-cycle; needs FP64 PCG vectors (pcg_vectors = 0) */

typedef struct vflip_learned_stats {
  int fallback;          /* 1: the learned iteration stalled; plain MGPCG solved from zero */
  int subspace;          /* vectors kept by the initial Ritz step (0-4) */
  double gamma[4];       /* Ritz coefficients of V(b), warm start, V(b) + coarse correction, previous pressure */
  double init_residual;  /* |b - A x0|_inf after the Ritz step */
  double net_ms;         /* network forward time */
} vflip_learned_stats;

/* Network grid for a fine grid and multigrid level: ceil(n / 2^level)
 * rounded up to a multiple of 8, per axis. */
int vflip_learned_grid(int ni, int nj, int nk, int level, int* X, int* Y, int* Z);

/* vflip_project with the learned preconditioner.  No reference counterpart:
 * an addition beside SmokeSolver3D::pcg_projection's solve, which stays the
 * plain path and the fallback.
 *   VFLIP_LEARNED_CAPTURE: plain MGPCG (same answer as vflip_project); the
 *     network grid (vflip_learned_grid at `level`) receives the features
 *     in2 = (s R^L rhs, R^L fluid) with s = 1 / |R^L rhs|_inf, the targets
 *     target2 = (s R^L p, s R^L (p - x1)) where p is the converged pressure
 *     and x1 plain PCG's first iterate, and weight = R^L fluid.
 *   VFLIP_LEARNED_SOLVE: the network maps the features to a warm-start
 *     pressure and a coarse correction (trilinear prolongation to the fine
 *     grid, scaled by vflip_unet_set_output_scale), each smoothed by
 *     VFLIP_LEARNED_SWEEPS(k) red-black Gauss-Seidel sweeps on A x = b (the
 *     correction after adding V(b)); the initial iterate minimises the
 *     energy error over span{V(b), warm start, V(b) + coarse correction}
 *     (plus the incoming pressure with VFLIP_LEARNED_PREV) (Ritz step), then
 *     flexible
 *     (Polak-Ribiere) PCG with the V-cycle runs to the same tolerance.  When
 *     the residual stalls (less than 2x reduction over two iterations, or
 *     NaN) plain MGPCG restarts from zero.  stats->vcycles counts every
 *     V-cycle, the Ritz step's and a fallback's included. */
int vflip_project_learned(vflip_ctx* ctx, vflip_unet* net, int mode, int level, int ni, int nj, int nk, float h,
                          float U_in, const float* nodal_phi, const int8_t* bdesc, const float* us, const float* vs,
                          const float* ws, float* u, float* v, float* w, double* pressure, double tolerance_factor,
                          int max_iterations, float* sample_in2, float* sample_target2, float* sample_weight,
                          vflip_solve_stats* stats, vflip_learned_stats* lstats);

/* ---- batched solves ---------------------------------------------------------- */

/* One Poisson system of a batch: the symmetric 7-point operator (diag, +x,
 * +y, +z couplings, FP64, as vflip_amgpcg_solve takes it), its rhs and the
 * result array, all device pointers. */
typedef struct vflip_system {
  int ni, nj, nk;
  const double *diag, *xp, *yp, *zp;
  const double* rhs;
  double* result;
} vflip_system;

#define VFLIP_BATCH_GRAPH 0 /* one CUDA graph: each system's PCG loop a device-side while node, systems in parallel */
#define VFLIP_BATCH_LOOP 1  /* one system after another (vflip_amgpcg_solve per system) */
#define VFLIP_BATCH_PERSISTENT 2 /* one persistent cooperative kernel over a (system, level, chunk) work list, in a
                                    CUDA graph (FP32/MIXED contexts; FP64 runs VFLIP_BATCH_GRAPH) */

/* Solves many independent systems of uneven sizes with the context's MGPCG
 * (same hierarchy, smoother, tolerance test and precision as
 * vflip_amgpcg_solve).  VFLIP_BATCH_GRAPH builds every system's hierarchy,
 * then captures the batch into one CUDA graph and launches it once: per
 * system a parallel branch whose PCG iterations run in a conditional while
 * node whose condition a kernel sets from the device-side scalars, so no
 * iteration returns to the host.  VFLIP_BATCH_PERSISTENT builds the
 * hierarchies the same way, then runs every system's PCG loop in ONE launch
 * of a persistent cooperative kernel (captured in a graph): each phase of
 * the V-cycle and of the PCG step is a work list of (system, chunk) items
 * taken by all resident CTAs, grid barriers between dependent phases, the
 * coarsest levels one CTA per system; systems leave the loop as they
 * converge.  Same stopping test and per-cell arithmetic; its reductions are
 * grouped per item, so its iterates agree with graph mode's to rounding.
 * Returns 0 when every system converged, 1
 * otherwise; stats[i] per system (solve_ms = the whole call, set-up
 * included; vflip_last_ms = the graph launch alone in graph mode).  No reference
 * counterpart (the reference solves one system per AMGPCGSolve call,
 * SS/AlgebraicMultigrid.h:189-301). */
int vflip_batched_solve(vflip_ctx* ctx, int nsys, const vflip_system* systems, double tolerance_factor,
                        int max_iterations, int mode, vflip_solve_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* VFLIP_H */
