/*
 * apcloud_gpu.h - C ABI of the B200 (sm_100a) AP-Cloud gravity step.
 *
 * One context owns one particle set resident in GPU memory and runs the reference's
 * per-timestep gravity path on it:
 *   octree build -> computational-particle selection -> GFD density + Laplacian
 *   stencils -> density and potential GMRES solves -> differentiation ->
 *   interpolation to particles + kick -> drift.
 *
 * The entry points replace these reference interfaces (paths relative to the
 * reference project root):
 *   apc_create / apc_set_particles   Physical_particle + Mover/Solver construction and
 *                                     setters (particle.h:5-21, mover.h:31-40,
 *                                     solver.h:53-60, controller.cpp:75-104)
 *   apc_select                        Mover::select_computational_particles
 *                                     (mover.cpp:17-49): Octree(...) (octree.h:224) +
 *                                     Octree::select_computational_particles_2to1_3d
 *                                     (octree.h:251, octree.cpp:1050-3001)
 *   apc_solve                         Solver::solve (solver.h:62, solver.cpp:382-454)
 *   apc_move_velocity                 Mover::move_velocity (mover.h:42, mover.cpp:51-89)
 *                                     incl. Octree::interpolation_from_node_to_particle_2to1_3d
 *                                     (octree.h:250, octree.cpp:3003-3031)
 *   apc_move_position                 Mover::move_position (mover.h:41, mover.cpp:91-121)
 *   apc_get_cells / apc_get_fields    the Computational_particle arrays
 *                                     (particle.h:23-53) the reference fills
 *
 * Conventions: every call returns an apc_status (0 = success; never exit()).
 * Host pointers are caller-owned; device buffers are owned by the context.  Each
 * context issues its work on CUDA streams of its own (its main stream, plus a copy stream
 * and a stream for the multigrid hierarchy that the main stream waits for); a context is
 * not thread-safe, distinct contexts are independent.
 */
#ifndef APCLOUD_GPU_H
#define APCLOUD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum apc_status {
  APC_OK = 0,
  APC_ERR_INVALID_ARG = -1,  /* bad size, pointer or parameter */
  APC_ERR_CUDA = -2,         /* a CUDA runtime call failed (see apc_last_error) */
  APC_ERR_OUT_OF_MEMORY = -3,
  APC_ERR_ORDER = -4,        /* phase called before its inputs exist (e.g. solve before select) */
  APC_ERR_NMAX = -5,         /* selection exceeded the temp-node budget even after doubling it
                                to the reference's 1e6 cap (mover.cpp:20,36-41 returns -1) */
  APC_ERR_STENCIL = -6,      /* GFD neighbour search failed where the reference exit()s:
                                too few neighbours after 5 expansions (solver.cpp:544-550) or
                                more candidates than the search buffers hold */
  APC_ERR_RANK = -7,         /* rank-deficient GFD least-squares system (solver.cpp:107-115) */
  APC_ERR_NOT_FINITE = -8,   /* NaN/Inf particle coordinates */
  APC_ERR_UNSUPPORTED = -9,
  APC_ERR_TIMEOUT = -10      /* a bounded device-side wait gave up */
} apc_status;

typedef enum apc_precision {
  APC_PREC_FP64 = 0,  /* FP64 GMRES with the reference's semantics: GMRES(restart) + Jacobi */
  APC_PREC_MIXED = 1, /* FP32 SpMV/Krylov inside an FP64 iterative-refinement loop */
  APC_PREC_FP64_MULTIGRID = 2, /* the mixed path's solver with every vector and operator in FP64:
                                 restarted (F)GMRES on the Jacobi-scaled systems, the potential
                                 right-preconditioned by the same octree multigrid, each cycle
                                 restarted from the true FP64 residual; same stopping test */
  APC_PREC_MIXED_VCYCLE = 3 /* the potential by FP64_MULTIGRID's FP64 FGMRES with the V-cycle
                               preconditioner in FP32 (hierarchy and smoothing sweeps); the density
                               as in MIXED (FP32 GMRES corrections in FP64 refinement); same
                               stopping test */
} apc_precision;

typedef struct apc_config {
  int n_particles;       /* Physical_particle::size */
  int depth;             /* MaxOctreeLevel: key bits = 3*depth, 1 <= depth <= 21 */
  int bc;                /* 1 periodic, 0 non-periodic (Periodic) */
  double box[6];         /* BoundingBox_min_x, max_x, min_y, max_y, min_z, max_z */
  double gfd_c;          /* CellSizeParameter: refine while n*h^2 > c */
  int lm;                /* NumberOfNeighbors: GFD stencil size, 10 <= lm <= 32 */
  int maxnc;             /* first temp-node budget (Mover::Set_maxnc; controller sets 10000).
                            The budget doubles on failure while below nmax_cap. */
  int nmax_cap;          /* budget cap: 1000000 reproduces mover.cpp:20; 0 = no cap */
  int gmres_restart;     /* -ksp_gmres_restart (PETSc default 30), 1..255 */
  double gmres_rtol;     /* -ksp_rtol */
  double gmres_atol;     /* -ksp_atol */
  double gmres_dtol;     /* -ksp_divtol */
  int gmres_max_it;      /* -ksp_max_it */
  int precision;         /* apc_precision */
  int mixed_restart;     /* inner restart of both multigrid-path solves (0 = 16 for the density solve and
                            the multigrid potential solve, 30 for the potential without multigrid),
                            at most 31 */
  double mixed_inner_rtol; /* FP32 inner solve relative tolerance (0 = 1e-3 with multigrid, 1e-5 without) */
  int device;            /* CUDA device ordinal */
  int mixed_precond;     /* APC_PREC_MIXED / APC_PREC_FP64_MULTIGRID potential solve: APC_PRECOND_JACOBI
                            or APC_PRECOND_MULTIGRID */
  int mg_sweeps;         /* multigrid: Jacobi sweeps before and after each coarse correction (0 = 2) */
  double mg_omega;       /* multigrid: Jacobi damping (0 = 0.95) */
  double mg_alpha;       /* multigrid: coarse-correction over-scaling (0 = 1.8) */
  int mg_reorth;         /* multigrid FGMRES: 1 = classical Gram-Schmidt twice, 0 = once (default) */
  int warm_start;        /* mixed path: start both solves from the previous step's solution at the
                            same octree cells (1) or from zero (0, default); the stopping test stays
                            rtol ||D^-1 b||.  At 128^3 and a < 0.1 it saves ~1 of 20 iterations */
  int mixed_solve_graphs; /* APC_PREC_MIXED / APC_PREC_FP64_MULTIGRID solves: 1 (default) = a CUDA graph
                            of per-phase kernels with conditional loop nodes; 0 = each solve is one
                            persistent cooperative kernel (refinement loop, (F)GMRES cycles and
                            V-cycles separated by grid barriers).  On a B200 at 128^3 the graph form
                            is faster (the barriers cost about what the launches they replace cost);
                            the queued batch mode uses the persistent form across boxes.
                            APC_PREC_MIXED_VCYCLE solves always run as graphs */
} apc_config;

enum { APC_PRECOND_JACOBI = 0, APC_PRECOND_MULTIGRID = 1 };

typedef struct apc_solve_stats {
  int density_its, potential_its;           /* inner iterations (FP32 ones in mixed mode; with the
                                               multigrid preconditioner, preconditioned iterations) */
  int density_reason, potential_reason;     /* PETSc KSPConvergedReason values */
  double density_rnorm, potential_rnorm;    /* final preconditioned residual norm */
  int density_refinements, potential_refinements; /* FP64 outer steps (mixed mode) */
  int mg_levels;                            /* multigrid levels of the last potential solve (0 = none) */
  int adjoint_density_its, adjoint_potential_its;       /* transposed solves of the last apc_solve_vjp */
  int adjoint_density_reason, adjoint_potential_reason;
} apc_solve_stats;

typedef struct apc_context apc_context;

/* Defaults: depth 21, periodic unit box, lm 17, maxnc 10000, nmax_cap 0, GMRES(30)
 * rtol 1e-10 atol 1e-50 dtol 1e5 max_it 10000, FP64; the mixed path's potential solve
 * uses the multigrid preconditioner. */
void apc_config_default(apc_config *cfg);
const char *apc_status_string(int status);
/* The message of the last failing call on this context (empty when none). */
const char *apc_last_error(const apc_context *ctx);

int apc_create(const apc_config *cfg, apc_context **out);
int apc_destroy(apc_context *ctx);

/* Particles: SoA FP64 host arrays of n_particles each.  apc_get_particles may be
 * given NULL for arrays the caller does not want; accelerations are those of the
 * last apc_move_velocity.  Particle order is the caller's order throughout.
 * apc_set_particles queues the copies and returns: from pinned host memory they run
 * asynchronously (the velocities on a copy stream beside the selection, as they are first
 * read by the kick), and the arrays must stay unchanged until the next phase call
 * (apc_select or apc_step) returns; pageable memory is staged during the call. */
int apc_set_particles(apc_context *ctx, const double *x, const double *y, const double *z,
                      const double *vx, const double *vy, const double *vz);
int apc_get_particles(apc_context *ctx, double *x, double *y, double *z, double *vx, double *vy,
                      double *vz, double *ax, double *ay, double *az);
/* Same with device pointers (n_particles doubles each, on the context's device). */
int apc_set_particles_device(apc_context *ctx, const double *x, const double *y, const double *z,
                             const double *vx, const double *vy, const double *vz);
int apc_get_particles_device(apc_context *ctx, double *x, double *y, double *z, double *vx,
                             double *vy, double *vz);

/* ---- phases, in Controller::solve order (controller.cpp:133-197) ---- */

/* Octree build + selection.  *n_cells = nc + nv + nb, the reference's return value. */
int apc_select(apc_context *ctx, int *n_cells);
/* GFD assembly, density solve, potential solve, differentiation.  c_dens, c_pot,
 * c_field are the constants of Solver::Set_Constant_For_* (controller.cpp:184-186). */
int apc_solve(apc_context *ctx, double c_dens, double c_pot, double c_field);
/* Interpolation + kick v += a c_vel dt; *max_dv = max |a| c_vel dt (may be NULL). */
int apc_move_velocity(apc_context *ctx, double dt, double c_vel, double *max_dv);
/* Drift x = wrap(x + v c_pos dt); *max_dx = max |v| c_pos dt (may be NULL). */
int apc_move_position(apc_context *ctx, double dt, double c_pos, double *max_dx);

/* One whole step {select; solve; move_velocity; move_position} with the constants of
 * controller.cpp:182-186 for time t and step dt.  The interpolation, kick and drift run
 * as one fused pass over the particles, bit-identical to apc_move_velocity followed by
 * apc_move_position.  Outputs may be NULL. */
typedef struct apc_step_params {
  double dt, c_dens, c_pot, c_field, c_vel, c_pos;
} apc_step_params;
int apc_step(apc_context *ctx, const apc_step_params *p, int *n_cells, double *max_dv,
             double *max_dx);

/* Wait for all work of the context. */
int apc_synchronize(apc_context *ctx);

/* ---- results of the last select / solve (parity and diagnostics) ---- */

int apc_get_cell_counts(apc_context *ctx, int *nc, int *nv, int *nb, int *n_neigh24);
/* Computational_particle arrays in the reference's output order.  first[i] of a cell
 * holding no particle is the sorted position where its particles would start. */
int apc_get_cells(apc_context *ctx, double *x, double *y, double *z, double *cell_length,
                  int *first, int *count, int *type, int *first_neigh, int *number_neigh,
                  int *neigh24);
/* Octree location code of every cell: (1 << 3*level) | Morton prefix. */
int apc_get_cell_codes(apc_context *ctx, uint64_t *codes);
/* Sorted Morton keys and the caller's particle index for each (octree.cpp:131-148). */
int apc_get_keys(apc_context *ctx, uint64_t *keys, int *index);
/* numnodes[0..depth]: octree node count per level (octree.cpp:174-191). */
int apc_get_octree_levels(apc_context *ctx, int *numnodes);
/* Density, Potential and p_x..p_yz (9 per cell, in that order) of cells 0..nc+nv-1. */
int apc_get_fields(apc_context *ctx, double *density, double *potential, double *deriv9);
/* GFD stencil of each cell: lm neighbour indices and distances, in search order (either
 * pointer may be NULL).  The distances are not kept by the step: asking for them computes
 * them from the indices on the device, as the least squares do, and needs a device buffer
 * of lm doubles per cell. */
int apc_get_stencils(apc_context *ctx, int *idx, double *dist);
int apc_get_solve_stats(apc_context *ctx, apc_solve_stats *stats);
/* Matrix A1 (which = 0) or A2 (which = 1) in CSR, columns sorted per row.  Call with
 * rowptr == NULL to get *n and *nnz first. */
int apc_get_matrix(apc_context *ctx, int which, int *n, int *nnz, int *rowptr, int *col,
                   double *val);

/* Number of kernels this context has launched since creation. */
int64_t apc_kernel_launches(const apc_context *ctx);

/* Counters of the GMRES kernel (the dominant kernel) since the last reset.
 * krylov_bytes follows the algorithmic model: per Arnoldi step
 * W*(S+4) + (2*j + 6)*S bytes per row for basis index j, where W is the ELL width and
 * S the vector word size.  A CGS2 step adds (j + 3)*S.  Each restart adds
 * W*(S+4) + 3*S and each solution update (j + 2)*S. */
typedef struct apc_profile {
  int64_t krylov_launches;
  int64_t krylov_iterations;
  double krylov_ms;      /* summed device time of those launches (CUDA events) */
  double krylov_bytes;   /* algorithmic bytes of those launches */
  double select_ms, solve_ms, move_ms;  /* summed phase device times */
  int64_t steps;         /* completed solve phases */
  double step_ms;        /* summed device time from each select to the next move_position */
  double gfd_ms;         /* summed device time of the GFD stencil + assembly kernel */
  double mg_build_ms;    /* summed time to build multigrid hierarchies (incl. host work) */
  double mg_solve_ms;    /* summed time of the multigrid-preconditioned FGMRES solves */
  int64_t mg_iterations; /* their FGMRES iterations */
  double assemble_ms;    /* summed device-timeline span of GFD assembly (stencils, matrices, rhs) */
  double density_ms;     /* ... of the density solve */
  double potential_ms;   /* ... of the potential solve (incl. hierarchy build and capture) */
  int64_t graph_instantiations;  /* solve graphs instantiated */
  int64_t graph_updates;         /* solve graphs updated in place from a new capture */
  int64_t sort_retries;  /* selections that went deeper than the particle sort and were redone
                            after a sort over every key bit */
  double mg_bytes;       /* algorithmic bytes of the multigrid-preconditioned solves counted in
                            mg_solve_ms: every array a phase must read or write, once per phase
                            (ELL values + columns, vectors, aggregation maps), summed over the
                            V-cycles, Arnoldi steps and FP64 refinement steps that ran */
} apc_profile;
int apc_get_profile(apc_context *ctx, apc_profile *out);
int apc_reset_profile(apc_context *ctx);

/* Interpolation + kick (the work of apc_move_velocity) on caller-owned device buffers,
 * for callers that cannot allocate device memory: embedders whose framework owns all
 * device memory through its own allocator, or loops that cannot afford the device-wide
 * synchronisation of cudaMalloc / cudaFree.  No counterpart in the reference: it has no
 * GPU code and no caller with this constraint.
 *
 * This call allocates nothing.  Its scratch (particle -> cell map, max-change
 * accumulator) is a fixed 4 MiB + 256 B array inside the library that every GPU loading
 * the library keeps until the process exits, so n_particles may not exceed
 * APC_NOALLOC_MAX_PARTICLES (larger sizes return APC_ERR_INVALID_ARG).  The first call
 * on a device looks up the array's device address (once per device) and should come
 * before any stream capture; that address is kept for the life of the process, so the
 * call must not be used on a device again after cudaDeviceReset there.  All calls share
 * the one array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  Each call resets the parts of the
 * scratch that must start cleared.
 *
 * Inputs, all device pointers on the current device: particles x, y, z in cell order
 * (cell i owns particles first[i] .. first[i]+count[i]-1); cell centres cx, cy, cz;
 * deriv9 = p_x p_y p_z p_xx p_yy p_zz p_xy p_xz p_yz per cell.  In/out: vx, vy, vz
 * (v += a c_vel dt).  Out: ax, ay, az; *max_dv (host, may be NULL) as apc_move_velocity.
 * The cell ranges must cover every particle exactly once: a range outside
 * [0, n_particles), overlapping ranges or an uncovered particle return
 * APC_ERR_INVALID_ARG, and then vx..az are left as they were.
 * stream: a cudaStream_t, or NULL for the default stream; the call returns after the
 * stream has finished its work. */
#define APC_NOALLOC_MAX_PARTICLES (1 << 20)
int apc_move_velocity_noalloc(int n_particles, int n_cells, const int *first, const int *count,
                              const double *cx, const double *cy, const double *cz,
                              const double *deriv9, const double *x, const double *y,
                              const double *z, double *vx, double *vy, double *vz, double *ax,
                              double *ay, double *az, double dt, double c_vel, double *max_dv,
                              void *stream);

/* Apply the PETSc KSP command-line options that the reference's runs pass to both solves
 * (KSPSetFromOptions, solver.cpp:202, 275; run lines in Makefile:30-32): -ksp_gmres_restart,
 * -ksp_rtol, -ksp_atol, -ksp_divtol, -ksp_max_it.  Other arguments are ignored, as PETSc
 * ignores options it does not use.  A restart above 255 returns APC_ERR_UNSUPPORTED (the
 * FP64 GMRES kernel keeps at most 255 basis vectors; the reference's production runs use
 * 200); a malformed value APC_ERR_INVALID_ARG. */
int apc_config_from_options(apc_config *cfg, int argc, const char *const *argv);

/* Adaptive time step (ADAPTIVE_TIME_STEP, controller.cpp:146-164), after apc_select:
 * max_density = max over the cells of n_p / h^3, reduced on the device in the reference's
 * operation order; dt = 0.05 delta_a / max_density^(1/2), at most delta_a (the caller
 * still clips t + dt to the end time, controller.cpp:168-169). */
int apc_max_cell_density(apc_context *ctx, double *max_density);
int apc_adaptive_dt(apc_context *ctx, double delta_a, double *dt);

/* Device time (ms) of the last select / solve / move phases, from CUDA events. */
int apc_get_phase_times(apc_context *ctx, double *select_ms, double *solve_ms, double *move_ms);

/* ---- diagnostics (no counterpart in the reference, which has no GPU code) ---- */

/* The compute capability the library's device code was built for, as the runtime loaded
 * it on `device` (cudaFuncGetAttributes: 100 = sm_100) and the PTX version behind it. */
int apc_device_code_version(int device, int *binary_version, int *ptx_version);

/* Self-check of the library's bounded device waits (the grid barrier of the persistent
 * GMRES kernel).  Two blocks are launched on `device`; one leaves without arriving at
 * the barrier, so the other's wait runs out after spin_limit polls (each a ~64 ns sleep;
 * 1 <= spin_limit <= 2^24) and it raises the error and abort flags and returns, as the
 * solver kernels do.  Returns APC_ERR_TIMEOUT when the wait gave up (the designed
 * outcome), APC_OK if the barrier completed.  The device stays usable either way. */
int apc_check_bounded_wait(int device, int spin_limit);

/* ---- derivatives ----
 * The reference computes no derivatives.  These entry points are the reverse mode of
 * the Controller step sequence (controller.cpp:88-208) with the octree, the selected
 * cells and their particle counts held fixed.  Under that assumption the cell fields of
 * a step do not depend on the positions (the density is n_p / h^3, solver.cpp:116-172),
 * and the Jacobian of the interpolated acceleration a = g + H (x - x_c)
 * (octree.cpp:3003-3031) is the cell's Hessian H. */

/* Per-particle Hessian (xx, yy, zz, xy, xz, yz) of the cell each particle was kicked in
 * by the last apc_move_velocity; device arrays of n_particles, caller order. */
int apc_get_hessians_device(apc_context *ctx, double *hxx, double *hyy, double *hzz, double *hxy,
                            double *hxz, double *hyz);

/* Reverse of one kick + drift: given the cotangents cot = (x, y, z, vx, vy, vz) of the
 * state after the step (device, caller order), overwrite them with those of the state
 * before it.  hess: the step's per-particle Hessians (apc_get_hessians_device);
 * kdt = C_vel dt, ddt = C_pos dt.  stream: cudaStream_t or NULL; returns when done. */
int apc_vjp_kick_drift(int n_particles, const double *const hess[6], double kdt, double ddt,
                       double *const cot[6], void *stream);

/* Re-solve the fields of the current cells for another density right-hand side
 * rhs_dev (device, M = nc + nv values in cell order; the reference's is n_p / h^3 C_dens,
 * solver.cpp:116-172), with the constants of the last apc_solve: density solve,
 * potential rhs, potential solve and differentiation (solver.cpp:182-362).  The
 * context's fields are replaced. */
int apc_fields_from_rhs(apc_context *ctx, const double *rhs_dev);

/* Vector-Jacobian product of the solve phase with respect to its density right-hand side:
 * given g_deriv (device, M x 9, the cotangent of the 9 field derivatives per cell),
 * write to g_rhs (device, M) the cotangent of the density rhs.  The transposed
 * differentiation stencil is applied, then FP64 GMRES on A2^T, the transposed mean
 * subtraction and FP64 GMRES on A1^T (the transposes are built from the current ELL
 * matrices; GMRES settings from the config).  g_rho / g_phi (optional, device, M)
 * receive the intermediate cotangents of the density and the potential.  Periodic boxes
 * only. */
int apc_solve_vjp(apc_context *ctx, const double *g_deriv, double *g_rhs, double *g_rho, double *g_phi);

typedef struct apc_trajectory {
  int n_steps;                   /* Controller steps after the start */
  const apc_step_params *steps;  /* one per step */
  double start_dt, start_c_pos;  /* the initial half drift: dt/2 and C_pos(start_a) */
  int checkpoint_every;          /* forward states kept every k steps, k >= 1 */
} apc_trajectory;

/* Vector-Jacobian product of a whole trajectory: select + half drift, then n_steps
 * apc_step calls, from the initial state state0 = (x, y, z, vx, vy, vz) (device, caller
 * order).  On entry cot holds the cotangents of the final state; on return those of
 * state0.  statef (optional, device) receives the final state.  The forward pass keeps
 * the state every checkpoint_every steps; the backward pass reruns each segment to
 * record its Hessians (bit-identical to the forward run) and applies the reverse steps.
 * Memory: 6 n doubles per checkpoint and per step of a segment. */
int apc_trajectory_vjp(apc_context *ctx, const apc_trajectory *t, const double *const state0[6],
                       double *const cot[6], double *const statef[6]);

/* ---- batches of independent boxes ----
 * The reference runs one box per process (test.cpp:16-80); it has no batched
 * interface.  A batch owns one context per box (each with its own stream) and steps
 * them together.  Each box's apc_step (controller.cpp:133-197, the same code path as a
 * single context) runs as a fiber on one of a few host threads, boxes dealt largest
 * first.  A fiber that waits on the GPU yields to the next box, so the GPU overlaps
 * the kernels of many small boxes.  Per-box results are those of the single-box path. */
typedef struct apc_batch apc_batch;

/* Create n_boxes contexts from cfgs[0..n_boxes-1] (all on cfgs[i].device), stepped by
 * n_workers host threads (0 = min(n_boxes, 16)), each running its boxes as fibers. */
int apc_batch_create(const apc_config *cfgs, int n_boxes, int n_workers, apc_batch **out);
int apc_batch_destroy(apc_batch *b);
int apc_batch_size(const apc_batch *b);

/* The context of box i: use it for particles I/O, selection, results and profiles.
 * Do not use it from another thread while apc_batch_step runs. */
apc_context *apc_batch_context(apc_batch *b, int box);

/* One step of every box: select, solve, kick and drift with params[i] for box i.
 * status[i] (optional) receives box i's apc_status; the call returns the first
 * non-zero status, or APC_OK.  max_dv / max_dx (optional, n_boxes each) receive the
 * boxes' kick and drift maxima. */
int apc_batch_step(apc_batch *b, const apc_step_params *params, int *status, double *max_dv,
                   double *max_dx);

/* How a batch step runs the boxes' multigrid solves.
 *   APC_BATCH_SOLVE_PER_BOX (default): each box's step runs whole in its fiber, its solves
 *     as its own persistent kernels; per-box results are those of a lone context, bit for bit.
 *   APC_BATCH_SOLVE_QUEUED: the step runs in three parts over all boxes - selection, assembly
 *     and the density solve's set-up; the potential rhs and the potential solve's set-up;
 *     differentiation, kick and drift - and between the parts ONE cooperative kernel runs
 *     every box's prepared solve: its block groups take boxes from a device work queue,
 *     largest first, and solve each with group-local barriers.  Per-box results meet the
 *     same stopping test as a lone context's (the sums run over other block counts, so they
 *     agree to the solver's tolerance, not bit for bit).  Boxes on the FP64 GMRES path
 *     (APC_PREC_FP64) solve at once in their fibers either way. */
enum { APC_BATCH_SOLVE_PER_BOX = 0, APC_BATCH_SOLVE_QUEUED = 1 };
int apc_batch_set_solve_mode(apc_batch *b, int mode);
/* Device time (ms) of the last step's two queued solve launches (0 per box). */
float apc_batch_solve_ms(const apc_batch *b);

#ifdef __cplusplus
}
#endif
#endif /* APCLOUD_GPU_H */
