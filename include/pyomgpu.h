/*
 * pyomgpu.h -- C ABI of the B200 external-mode (barotropic) solver for pyOM2.
 *
 * Drop-in for the routines pyOM2's f2py module binds for this path
 * (py_src/Makefile:15-47 builds them into ``pyOM_code``):
 *
 *   reference routine (file:line)                      replaced by
 *   ---------------------------------------------------------------------------
 *   make_coeff_streamfunction  solve_streamfct.f90:123  pyomgpu_ctx_create (operator kept, like the SAVE'd cf)
 *   make_coeff_surf_press      solve_pressure.f90:87    pyomgpu_ctx_create (second operator)
 *   make_inv_sfc               solve_streamfct.f90:381  pyomgpu_set_islands / pyomgpu_streamfunction_init
 *   congrad_streamfunction     solve_streamfct.f90:153  pyomgpu_congrad_streamfunction
 *   congrad_surf_press         solve_pressure.f90:137   pyomgpu_congrad_surf_press
 *   apply_op                   solve_pressure.f90:254   pyomgpu_apply_op
 *   dot_sfc/absmax_sfc         solve_streamfct.f90:331-362 (fused into the CG kernels)
 *   dot_sfp/absmax_sfp         solve_pressure.f90:277-311  (fused into the CG kernels)
 *   streamfunction_init        streamfct_init.f90:7     pyomgpu_streamfunction_init (+ _get_islands)
 *   isleperim                  island_module.f90:7      pyomgpu_isleperim
 *   line_integral              streamfct_init.f90:311   pyomgpu_line_integral
 *   solve_streamfunction       solve_streamfct.f90:10   pyomgpu_solve_streamfunction
 *   solve_pressure             solve_pressure.f90:10    pyomgpu_solve_pressure
 *   make_coeff_non_hydro       non_hydrostatic.f90:70   pyomgpu_nh_create (operator kept, like the SAVE'd cf)
 *   congrad_non_hydro          non_hydrostatic.f90:146  pyomgpu_congrad_non_hydro
 *   apply_op_3D                non_hydrostatic.f90:247  pyomgpu_apply_op_3d
 *   dot_3D/absmax_3D           non_hydrostatic.f90:279-322 (fused into the CG kernel)
 *   solve_non_hydrostatic      non_hydrostatic.f90:5    pyomgpu_solve_non_hydrostatic
 *
 * Array conventions: every 2-D field has the Fortran extents of
 * main_module.f90 for one PE, (1-onx:nx+onx, 1-onx:ny+onx) with onx = 2, in
 * Fortran (column-major) order, leading dimension nx+4 -- exactly the buffers
 * f2py exposes.  3-D fields append nz, 4-D fields append (nz, 3) time levels.
 * Island arrays boundary/line_dir are (nisle, max_boundary, 2) int32 in
 * Fortran order with Fortran index values.
 *
 * Pointers marked "host or device" may point to either; the library detects
 * host memory with cudaPointerGetAttributes and stages it through device
 * buffers owned by the context.  Grid inputs to pyomgpu_ctx_create are host
 * pointers.  The full-step entry points take device pointers.
 *
 * Errors never abort the process (the reference calls halt_stop,
 * parallel_none.f90:51-59): every entry point returns a status code and
 * pyomgpu_last_error() gives a message.  A context is used by one host thread
 * at a time; all work is ordered on the stream passed in.
 */
#ifndef PYOMGPU_H
#define PYOMGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pyomgpu_ctx pyomgpu_ctx;
typedef void* pyomgpu_stream; /* a cudaStream_t; NULL = legacy default stream */

/* ---- status codes --------------------------------------------------------- */
#define PYOMGPU_OK 0
#define PYOMGPU_MAXITER 1   /* max iterations exceeded (solve_streamfct.f90:303) */
#define PYOMGPU_DIVERGED 2  /* divergence test fired (solve_streamfct.f90:236) */
#define PYOMGPU_NAN 3       /* estimated error is NaN (solve_streamfct.f90:322) */
#define PYOMGPU_TIMEOUT 4   /* a device-side grid barrier wait ran out */
#define PYOMGPU_SINGULAR 5  /* island system singular (DGESV info != 0, solve_streamfct.f90:82) */
#define PYOMGPU_EINVAL -1
#define PYOMGPU_ECUDA -2
#define PYOMGPU_ENOMEM -3
#define PYOMGPU_EISLAND -4 /* island labelling / perimeter tracing failed */
#define PYOMGPU_ESTATE -5  /* call needs state the context does not have yet */

/* operators held by a context */
#define PYOMGPU_OP_STREAMFUNCTION 0 /* solve_streamfct.f90:123-148 */
#define PYOMGPU_OP_SURF_PRESS 1     /* solve_pressure.f90:87-131 */

/* arithmetic of pyomgpu_solve_rtol */
#define PYOMGPU_PREC_F64 64 /* FP64 Jacobi-PCG */
#define PYOMGPU_PREC_F32 32 /* FP32 PCG with FP64 dot products inside FP64 iterative refinement */

/* Geometry and operator inputs: the main_module arrays the solve reads
 * (main_module.f90:115-121,185-192).  All host pointers. */
typedef struct pyomgpu_grid {
  int32_t nx, ny;      /* interior points (serial: is_pe=1, ie_pe=nx) */
  int32_t onx;         /* halo width; must be 2 */
  int32_t enable_cyclic_x, enable_cyclic_y;
  int32_t enable_free_surface; /* adds -maskT/(grav dt^2) to the surf_press diagonal */
  double grav, dt_mom;         /* only for the free-surface diagonal */
  const double *dxt, *dxu;     /* [nx+4] */
  const double *dyt, *dyu;     /* [ny+4] */
  const double *cost, *cosu;   /* [ny+4] */
  const double *hur, *hvr;     /* streamfunction operator */
  const double *hu, *hv;       /* surface-pressure operator (may be NULL if unused) */
  const double *maskT_top;     /* maskT(:,:,nz) (surface pressure; may be NULL) */
  const double *maskU_top, *maskV_top; /* maskU/maskV(:,:,nz) for island integrals (may be NULL) */
} pyomgpu_grid;

/* Island description as produced by streamfunction_init (streamfct_init.f90:87-93). */
typedef struct pyomgpu_islands {
  int32_t nisle;
  int32_t max_boundary;
  const int32_t* boundary;    /* (nisle, max_boundary, 2) host */
  const int32_t* line_dir;    /* (nisle, max_boundary, 2) host */
  const int32_t* nr_boundary; /* (nisle) host */
} pyomgpu_islands;

/* Result of one solve. */
typedef struct pyomgpu_solve_info {
  int32_t iterations;       /* congr_itts (inner iterations summed for refinement) */
  int32_t converged;        /* the logical ``converged`` of congrad_streamfunction */
  int32_t status;           /* PYOMGPU_* */
  int32_t outer_iterations; /* refinement sweeps (pyomgpu_solve_rtol F32) */
  double estimated_error;   /* the reference's estimated_error */
  double rel_residual;      /* FP64 ||b-Ax||/||b|| over the unknowns (solve_rtol only) */
  double device_ms;         /* device time of the CG kernel launch(es), CUDA events on the stream */
  int32_t kernel_launches;  /* kernels the call launched (solve_rtol; 1 = the CG kernel elsewhere) */
  int32_t fcg_iterations;   /* iterations of the flexible-CG phase (pyomgpu_solve_fcg), else 0 */
} pyomgpu_solve_info;

/* Model arrays of one time step (all DEVICE pointers, Fortran layout). */
typedef struct pyomgpu_state {
  int32_t nz;
  int32_t taum1, tau, taup1;    /* 1-based time levels */
  int32_t congr_max_iterations;
  int32_t congr_itts;           /* out */
  double dt_mom, AB_eps, grav, rho_0, congr_epsilon;
  const double *dzt, *dzw;      /* [nz] */
  const double *maskT, *maskU, *maskV; /* (nx+4,ny+4,nz) */
  const double* rho;            /* (nx+4,ny+4,nz,3) */
  double *u, *v, *du, *dv;      /* (nx+4,ny+4,nz,3) */
  const double *du_mix, *dv_mix;/* (nx+4,ny+4,nz) */
  double* p_hydro;              /* (nx+4,ny+4,nz) */
  double *psi, *dpsi;           /* (nx+4,ny+4,3) */
  double* dpsin;                /* (nisle,3), streamfunction only */
} pyomgpu_state;

/* Inputs and outputs of the momentum tendencies (momentum.f90:4-152) of a
 * hydrostatic configuration without turbulence closures (vertical viscosity
 * kappaM given, as the reference's kappaM_0 set-ups without TKE).  All
 * DEVICE pointers, Fortran layout with the module's halo; the 1-D grid
 * metrics dxt, dxu, dyt, dyu, cost, cosu come from the context. */
typedef struct pyomgpu_momentum {
  int32_t nz, taum1, tau, taup1;  /* 1-based time levels */
  int32_t coord_degree;           /* metric terms of momentum.f90:19-30 */
  int32_t enable_hor_friction, enable_hor_friction_cos_scaling, hor_friction_cospower;
  int32_t enable_bottom_friction, enable_implicit_vert_friction;
  double dt_mom, A_h, r_bot;
  const double *dzt, *dzw;        /* [nz] */
  const double* tantr;            /* [ny+4] */
  const double *maskT, *maskU, *maskV, *maskW; /* (nx+4,ny+4,nz) */
  const int32_t* kbot;            /* (nx+4,ny+4) */
  const double *coriolis_t, *area_t, *area_u, *area_v; /* (nx+4,ny+4) */
  const double *surface_taux, *surface_tauy;          /* (nx+4,ny+4) */
  const double* kappaM;           /* (nx+4,ny+4,nz) */
  double *u, *v, *w;              /* (nx+4,ny+4,nz,3); u, v(taup1) are the implicit friction's scratch */
  double *du, *dv;                /* (nx+4,ny+4,nz,3): du, dv(tau) written */
  double *du_mix, *dv_mix;        /* (nx+4,ny+4,nz) written */
} pyomgpu_momentum;

/* ---- library -------------------------------------------------------------- */
int32_t pyomgpu_version(void);
const char* pyomgpu_last_error(void);

/* Create a context for one grid on the current CUDA device: builds the
 * streamfunction operator (and the surface-pressure operator when hu/hv and
 * maskT_top are given) in device memory.  make_coeff_* of the reference is
 * run once and kept, like its SAVE'd cf (solve_streamfct.f90:172-180). */
int32_t pyomgpu_ctx_create(const pyomgpu_grid* grid, pyomgpu_ctx** out);
void pyomgpu_ctx_destroy(pyomgpu_ctx* ctx);

/* Device-side time limit of every grid-barrier wait (default 2 s). */
int32_t pyomgpu_set_sync_timeout(pyomgpu_ctx* ctx, double seconds);
/* Failure-detection test hook: when enabled, the next solver launch waits at
 * its first grid barrier for one block more than it launched, so every wait
 * runs into the time limit and the call returns PYOMGPU_TIMEOUT (no fault, the
 * context stays usable).  Cleared after that launch. */
int32_t pyomgpu_inject_barrier_stall(pyomgpu_ctx* ctx, int32_t enable);

/* CG kernel of the streamfunction solves (congrad_streamfunction,
 * solve_streamfunction, solve_rtol F64, the learned solver's fallback):
 * 1 = the tiled kernel (any grid; the one pyomgpu_autotune tunes),
 * 2 = the on-chip-resident kernel (one piece of the grid per SM, with the
 *     direction and face couplings in shared memory and the residual,
 *     solution and preconditioner in tensor memory for the whole solve;
 *     grids whose largest piece fits, about 1.04 M points on 148 SMs), with
 *     the reference's two reductions per iteration,
 * 3 = the same resident layout with one reduction per iteration (A p by
 *     recurrence and the reference's (p, Ap) by its exact bilinear expansion
 *     in products of the sweep before; the reference's stopping tests are
 *     evaluated one reduction later, on the same quantities),
 * 0 = automatic (2 wherever the grid fits: the reference's own recurrences;
 *     at 1440 x 720 3 runs on par with it).  PYOMGPU_EINVAL for 2 or 3 on a
 * grid that does not fit.  The surface-pressure solve always uses 1.
 * Reduction order and recurrences differ between the kernels: results
 * change at rounding level. */
int32_t pyomgpu_set_cg_kernel(pyomgpu_ctx* ctx, int32_t kernel);
/* Piece layout the resident kernel uses on this grid: pieces in x and y and
 * points per thread; PYOMGPU_EINVAL when the grid does not fit. */
int32_t pyomgpu_resident_layout(pyomgpu_ctx* ctx, int32_t* npx, int32_t* npy, int32_t* points_per_thread);
/* The same for the FP32 resident kernel that runs the correction solves of
 * pyomgpu_solve_rtol with PYOMGPU_PREC_F32 where the grid fits (FP32 fields
 * take half the on-chip memory, so grids up to twice the size fit; elsewhere,
 * or with set_cg_kernel 1, the pipelined tile kernel runs them). */
int32_t pyomgpu_resident_layout32(pyomgpu_ctx* ctx, int32_t* npx, int32_t* npy, int32_t* points_per_thread);
/* Diagnostics, no counterpart in the reference: one pyomgpu_solve_rtol (FP64)
 * in an instantiation of the resident kernel that records %globaltimer (ns)
 * at 18 phase boundaries of loop trips it0 .. it0+nit-1 in every block (the
 * same arithmetic and iterates).  out: host array of nblocks x nit x 18
 * words, [(block * nit + trip - it0) * 18 + phase]; phases: 0 sweep A start,
 * 1 direction in shared memory, 2 stencil and partials done, 3 after the
 * first block barrier, 4 after the second (alpha known), 5 residual updated,
 * 6 exchange records written, 7 after the first barrier of sweep B, 8
 * solution updated, 9 after the second (beta known, halo loaded); control
 * warp: 10/14 after the first barrier of reduction A/B, 11/15 its slot
 * published, 12/16 all slots acquired, 13/17 control step done.  nblocks
 * receives the block count (at most 160).  Zero words: phase not reached. */
int32_t pyomgpu_resident_trace(pyomgpu_ctx* ctx, const double* forc, double* sol, double rtol, int32_t it0,
                               int32_t nit, uint64_t* out, int32_t* nblocks, pyomgpu_solve_info* info,
                               pyomgpu_stream stream);

/* Autotuner of the solve kernel: times `iterations` iterations of the
 * Jacobi-PCG kernel on this grid (a fixed pseudo-random right-hand side) for
 * every tile shape tx x ty in {32,64,96,128} x {8,16,24,32} and every
 * co-resident grid size that changes the busiest block's tile count, and
 * keeps the fastest for all later streamfunction solves of the context
 * (congrad_streamfunction, solve_rtol F64, solve_streamfunction, the
 * learned solver's fallback).  Reduction order follows the tiling, so results
 * change at rounding level (iteration counts within one).  Outputs may be
 * NULL.  Not in the reference. */
int32_t pyomgpu_autotune(pyomgpu_ctx* ctx, int32_t iterations, int32_t* tile_x, int32_t* tile_y, int32_t* grid,
                         double* us_per_iteration, pyomgpu_stream stream);

/* ---- islands (streamfct_init.f90, island_module.f90) ------------------------ */
/* isleperim on a (imt,jmt) int map; map, nippts (>= mnisle entries) host.
 * Limits default to the reference's (mnisle 1000, maxipp 20000, maxq 10000)
 * when passed as 0. */
int32_t pyomgpu_isleperim(const int32_t* kmt, int32_t imt, int32_t jmt, int32_t cyclic, int32_t mnisle,
                          int32_t maxipp, int32_t maxq, int32_t* map, int32_t* nisle, int32_t* nippts);

/* Island labels and perimeters of streamfunction_init (streamfct_init.f90:35-267)
 * on the host, without the psin solves.  kbot is (nx+4, ny+4) host.  Call
 * first with boundary == NULL to get nisle and max_boundary, then with arrays
 * of (nisle, max_boundary, 2) / (nisle) entries. */
int32_t pyomgpu_island_boundaries(int32_t nx, int32_t ny, int32_t cyclic_x, const int32_t* kbot, int32_t mnisle,
                                  int32_t maxipp, int32_t maxq, int32_t* nisle, int32_t* max_boundary,
                                  int32_t* boundary, int32_t* line_dir, int32_t* nr_boundary);

/* The same result computed on the GPU (current device): connected-component
 * labelling by union-find with labels in the reference's scan order, and one
 * thread walking each island's coast.  kbot host or device.  Bit-identical to
 * pyomgpu_island_boundaries; the flood-fill queue limit maxq does not apply
 * (there is no queue).  Not in the reference. */
int32_t pyomgpu_island_boundaries_gpu(int32_t nx, int32_t ny, int32_t cyclic_x, const int32_t* kbot, int32_t mnisle,
                                      int32_t maxipp, int32_t maxq, int32_t* nisle, int32_t* max_boundary,
                                      int32_t* boundary, int32_t* line_dir, int32_t* nr_boundary,
                                      pyomgpu_stream stream);

/* Whole of streamfunction_init: land map from kbot (host), island labels,
 * perimeter tracing, one psin solve per island (batched on the GPU) and the
 * line_psin matrix (labelling and tracing as pyomgpu_island_boundaries_gpu).
 * Results stay in the context; read them with
 * pyomgpu_island_sizes / pyomgpu_get_islands. */
int32_t pyomgpu_streamfunction_init(pyomgpu_ctx* ctx, const int32_t* kbot, int32_t mnisle, int32_t maxipp,
                                    int32_t maxq, double congr_epsilon, int32_t congr_max_iterations,
                                    pyomgpu_stream stream);
/* momentum (momentum.f90:4-152) up to the external-mode solve, for the
 * hydrostatic case without closures: Coriolis and metric terms, surface wind
 * stress, momentum_advection (momentum_advection.f90:1-76), implicit
 * vertical friction with the given kappaM (vertical_friction.f90:109-226),
 * harmonic friction (harmonic_friction.f90:4-124) and linear bottom friction
 * (bottom_friction.f90:48-135), each as enabled in `m`.  Writes du, dv at
 * tau and du_mix, dv_mix on the interior points, bit for bit the reference's
 * serial arithmetic (the energy-dissipation diagnostics K_diss_* are not
 * formed).  The caller then runs pyomgpu_solve_streamfunction. */
int32_t pyomgpu_momentum_tendencies(pyomgpu_ctx* ctx, const pyomgpu_momentum* m, pyomgpu_stream stream);
/* The end of the reference's time step for u, v at `level`: their cyclic
 * halo copies (setcyclic_xyz, main.f90:114-117), then vertical_velocity
 * (vertical_velocity.f90:4-25, main.f90:147): w(:,:,:,level) from u, v at
 * `level`.  Uses m->u, m->v, m->w, m->maskW, m->dzt, m->nz only. */
int32_t pyomgpu_vertical_velocity(pyomgpu_ctx* ctx, const pyomgpu_momentum* m, int32_t level,
                                  pyomgpu_stream stream);

/* Stop of the psin solves of the next pyomgpu_streamfunction_init.  No
 * counterpart in the reference, which solves them with congrad_streamfunction
 * and its own stop (streamfct_init.f90:283): rtol = 0 (the default) keeps
 * that.  rtol > 0 solves each to ||res|| <= rtol ||res_0|| over the unknowns
 * instead (the forcing is zero) with the reference's stopping estimate off;
 * weighted = 1 then takes the inner products with the cell area dxu dyu cosu,
 * in which the operator A = D^-1 S is self-adjoint, so the iteration is
 * exact Jacobi-PCG on the symmetric S and converges where the reference's
 * Euclidean products stagnate (on grids whose cell area varies strongly,
 * e.g. 80S-80N).  PYOMGPU_EINVAL for rtol outside [0, 1). */
int32_t pyomgpu_set_psin_solve(pyomgpu_ctx* ctx, double rtol, int32_t weighted);
int32_t pyomgpu_island_sizes(pyomgpu_ctx* ctx, int32_t* nisle, int32_t* max_boundary);
/* Copies out boundary/line_dir/nr_boundary (host), psin (host or device,
 * (nx+4,ny+4,nisle)), line_psin (host, (nisle,nisle)) and the psin iteration
 * counts (host, nisle; may be NULL). */
int32_t pyomgpu_get_islands(pyomgpu_ctx* ctx, int32_t* boundary, int32_t* line_dir, int32_t* nr_boundary,
                            double* psin, double* line_psin, int32_t* psin_iterations, pyomgpu_stream stream);
/* Import islands computed elsewhere (e.g. by the Fortran streamfunction_init):
 * builds Z (make_inv_sfc).  psin (host or device) and line_psin (host) may be
 * NULL when only congrad_streamfunction is needed. */
int32_t pyomgpu_set_islands(pyomgpu_ctx* ctx, const pyomgpu_islands* isl, const double* psin,
                            const double* line_psin, pyomgpu_stream stream);

/* ---- solvers ---------------------------------------------------------------- */
/* congrad_streamfunction (solve_streamfct.f90:153-327): FP64 Jacobi-PCG with the
 * reference's stopping estimate, divergence test and s.As guard.  forc is
 * read, sol (in/out) is updated in place; both host or device. */
int32_t pyomgpu_congrad_streamfunction(pyomgpu_ctx* ctx, const double* forc, double* sol, double congr_epsilon,
                                       int32_t congr_max_iterations, pyomgpu_solve_info* info,
                                       pyomgpu_stream stream);

/* Allocation-free congrad_streamfunction.  No counterpart in the reference
 * (pyOM2 runs on the CPU and never meets this constraint).  For callers that
 * cannot call cudaMalloc: a host program whose device memory is fully claimed
 * by its own pool, code running where new device allocations are forbidden,
 * or a time loop that must not allocate (an allocation can synchronise the
 * device or fail under memory pressure mid-run).  It takes no context: the
 * grid (every pointer in `grid` a DEVICE pointer; hur/hvr and the six 1-D
 * metrics are read, the rest ignored), the island perimeter points bnd_i/bnd_j
 * (device int32, Fortran indices, nbnd of them: make_inv_sfc's Dirichlet
 * points), forc (device) and sol (device, in/out) are the only memory it
 * touches besides a static device array of PYOMGPU_NOALLOC_SCRATCH_BYTES that
 * the library holds on every GPU it is used on, until the process exits.  All
 * pointers must be memory of the current device (or managed memory).
 * Grids whose operator and work vectors exceed that array (about 1.0e6
 * padded points, e.g. 1000 x 1000) are rejected with PYOMGPU_EINVAL and a
 * message.  CUDA loads device code lazily, so the array and the solver's
 * kernels are placed on a device by the first call made there, which also
 * looks up the array's device address (cudaGetSymbolAddress): make that first
 * call at set-up, while device memory is free (it can fail with
 * PYOMGPU_ECUDA under memory pressure) and before any stream capture.  Later
 * calls take no device memory.  Every call reuses the same array and clears
 * what must start at zero; calls that overlap on the GPU (other streams or
 * host threads) race on it.  The call waits for `stream` before it returns,
 * because it reads the iteration count and status back to the host.
 * Results equal pyomgpu_congrad_streamfunction's on the same inputs. */
#define PYOMGPU_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int32_t pyomgpu_congrad_streamfunction_noalloc(const pyomgpu_grid* grid, const int32_t* bnd_i, const int32_t* bnd_j,
                                               int32_t nbnd, const double* forc, double* sol, double congr_epsilon,
                                               int32_t congr_max_iterations, pyomgpu_solve_info* info,
                                               pyomgpu_stream stream);

/* `count` congrad_streamfunction solves in ONE launch of a persistent
 * work-queue kernel.  Replaces the reference's one-after-another calls of
 * congrad_streamfunction (the psin loop, streamfct_init.f90:272-287, or a loop
 * over independent grids).  Solve k runs on ctx[k]'s grid and operator;
 * contexts may repeat (several right-hand sides on one grid) but must live on
 * one device.  forc[k] (read; forc or forc[k] NULL = zero forcing) and sol[k]
 * (in/out) are Fortran-layout, host or device.  Every solve keeps its own
 * scalars and follows congrad_streamfunction's control flow, so its
 * iterations, status and estimated_error are those of a separate call (dot
 * products are summed in another order).  rtol > 0 adds the stop of
 * pyomgpu_solve_rtol on the recursively updated residual and fills each
 * info's rel_residual with the FP64 true residual; congr_epsilon = 0 leaves
 * rtol as the only stop.  info: count entries or NULL; device_ms and
 * kernel_launches describe the whole call.  The work buffers live in ctx[0]
 * and grow to the largest batch it has run.  Returns the largest status.
 * Engine (pyomgpu_set_batch_kernel on ctx[0]): where every grid fits on chip,
 * on-chip-resident solves run side by side in one launch, each on its own set
 * of SMs, placed by list scheduling on the host; else the work-queue kernel
 * streams all solves through HBM in lockstep.  The rtol stop is relative to
 * ||forc||, or to the initial residual for a zero forcing. */
int32_t pyomgpu_congrad_streamfunction_batch(pyomgpu_ctx* const* ctx, int32_t count, const double* const* forc,
                                             double* const* sol, double congr_epsilon, int32_t congr_max_iterations,
                                             double rtol, pyomgpu_solve_info* info, pyomgpu_stream stream);

/* Engine of pyomgpu_congrad_streamfunction_batch calls owned by ctx (ctx[0]):
 * 0 automatic (resident groups where every grid fits on chip), 1 the
 * work-queue kernel, 2 resident groups (PYOMGPU_EINVAL from the batch call
 * when a grid does not fit).  No counterpart in the reference. */
int32_t pyomgpu_set_batch_kernel(pyomgpu_ctx* ctx, int32_t kernel);
/* Diagnostics of the last resident batch owned by ctx (ctx[0] of the call),
 * per solve in call order: device start and end (ms after the earliest
 * start, %globaltimer) and SMs used.  PYOMGPU_ESTATE when that batch had
 * another count or none ran on the resident engine.  Any output may be NULL. */
int32_t pyomgpu_batch_schedule(pyomgpu_ctx* ctx, int32_t count, double* start_ms, double* end_ms, int32_t* blocks);
/* The host planner of the resident batch on its own (no GPU work): `count`
 * jobs, job k needing blocks[k] of nsm blocks for est[k]; `tries` local-search
 * steps over the order.  Outputs (each may be NULL): rank (the order every
 * block runs its jobs in), planned start, the blocks of each job (gang,
 * count x nsm, ascending, padded with -1) and the planned makespan. */
int32_t pyomgpu_plan_batch(int32_t nsm, int32_t count, const int32_t* blocks, const double* est, int32_t tries,
                           int32_t* rank, double* start, int32_t* gang, double* makespan);
/* The piece cut of the resident kernel on its own (no GPU work): among the
 * cuts of an nx x ny grid into at most max_blocks pieces that fit in
 * smem_cap bytes of dynamic shared memory and in the worker threads at
 * points_per_thread (FP64: 4, 8 or 16; fp32: 16 or 32; 0: the smallest that
 * fits), the one with the least estimated iteration time, or with
 * least_block_time the least estimate x pieces (the densest cut of a batch
 * gang).  fp32: the FP32 instance of the mixed-precision correction solves.
 * out: npx, npy, the largest piece's w and h, and the points per thread;
 * est_ns: the estimate.  PYOMGPU_OK with out[0] = 0 when no cut fits.  No
 * counterpart in the reference. */
int32_t pyomgpu_plan_cut(int32_t nx, int32_t ny, int32_t max_blocks, int64_t smem_cap, int32_t points_per_thread,
                         int32_t least_block_time, int32_t fp32, int32_t* out, double* est_ns);

/* congrad_surf_press (solve_pressure.f90:137-249): FP64 CG with maskT-weighted
 * products.  psi is psi(:,:,taup1), in/out, host or device. */
int32_t pyomgpu_congrad_surf_press(pyomgpu_ctx* ctx, const double* forc, double* psi, double congr_epsilon,
                                   int32_t congr_max_iterations, pyomgpu_solve_info* info, pyomgpu_stream stream);

/* Solve A sol = forc (streamfunction operator, island perimeters Dirichlet)
 * until the FP64 true relative residual ||forc - A sol||_2/||forc||_2 over the
 * unknowns is <= rtol.  precision: PYOMGPU_PREC_F64 or PYOMGPU_PREC_F32.
 * Measurement entry point of the ms/solve metric; not in the reference. */
int32_t pyomgpu_solve_rtol(pyomgpu_ctx* ctx, const double* forc, double* sol, double rtol, int32_t precision,
                           int32_t max_iterations, pyomgpu_solve_info* info, pyomgpu_stream stream);

/* ---- operator utilities ------------------------------------------------------ */
/* res = A p over the interior, zero halo (apply_op, solve_pressure.f90:254-274). */
int32_t pyomgpu_apply_op(pyomgpu_ctx* ctx, int32_t op, const double* p, double* res, pyomgpu_stream stream);
/* The Jacobi inverse Z of make_inv_sfc (solve_streamfct.f90:381-422), Fortran layout. */
int32_t pyomgpu_get_inv_diag(pyomgpu_ctx* ctx, double* Z, pyomgpu_stream stream);
/* line_integral (streamfct_init.f90:311-377) of island isle (1-based). */
int32_t pyomgpu_line_integral(pyomgpu_ctx* ctx, int32_t isle, const double* uloc, const double* vloc, double* line,
                              pyomgpu_stream stream);

/* ---- one time step ------------------------------------------------------------ */
/* solve_streamfunction (solve_streamfct.f90:10-120) on device-resident model
 * arrays; islands must have been set up.  OBC (set_obc_streamfct) is not
 * supported. */
int32_t pyomgpu_solve_streamfunction(pyomgpu_ctx* ctx, pyomgpu_state* st, pyomgpu_solve_info* info,
                                     pyomgpu_stream stream);
/* solve_streamfunction split around its solve, so that any solver (the batch
 * kernel over ensemble members, pyomgpu_solve_rtol, pyomgpu_solve_fcg) can
 * take the place of congrad_streamfunction (solve_streamfct.f90:57):
 *   _begin: hydrostatic pressure and its gradient, the forcing (written to
 *           forc, a DEVICE (nx+4, ny+4) array; fpx/fpy stay in the context)
 *           and the first guess 2 dpsi(tau) - dpsi(taum1) in dpsi(:,:,taup1)
 *           (solve_streamfct.f90:24-56);
 *   _end:   dpsi(:,:,taup1) made cyclic, the island correction, psi and the
 *           3-D velocity update (:58-118).
 * begin + pyomgpu_congrad_streamfunction + end computes what
 * pyomgpu_solve_streamfunction does.  Stream-ordered; no synchronisation. */
int32_t pyomgpu_solve_streamfunction_begin(pyomgpu_ctx* ctx, pyomgpu_state* st, double* forc, pyomgpu_stream stream);
int32_t pyomgpu_solve_streamfunction_end(pyomgpu_ctx* ctx, pyomgpu_state* st, pyomgpu_stream stream);
/* solve_pressure (solve_pressure.f90:10-82) on device-resident model arrays. */
int32_t pyomgpu_solve_pressure(pyomgpu_ctx* ctx, pyomgpu_state* st, pyomgpu_solve_info* info,
                               pyomgpu_stream stream);

/* ---- non-hydrostatic pressure (non_hydrostatic.f90) --------------------------- */
/* Grid of the 3-D solve: main_module arrays, host pointers, Fortran order.
 * Masks hold only 0 and 1 (as calc_topo builds them, numerics.f90:187-249);
 * maskW(:,:,k) = min(maskT(:,:,k), maskT(:,:,k+1)) for k < nz. */
typedef struct pyomgpu_grid3d {
  int32_t nx, ny, nz;          /* nx >= 4, ny >= 1, nz >= 2 */
  int32_t onx;                 /* halo width; must be 2 */
  int32_t enable_cyclic_x, enable_cyclic_y;
  const double *dxt, *dxu;     /* [nx+4] */
  const double *dyt, *dyu;     /* [ny+4] */
  const double *cost, *cosu;   /* [ny+4] */
  const double *dzt, *dzw;     /* [nz] */
  const double *maskT, *maskU, *maskV, *maskW; /* (nx+4, ny+4, nz) */
} pyomgpu_grid3d;
typedef struct pyomgpu_nh pyomgpu_nh;

/* Builds the operator of make_coeff_non_hydro (non_hydrostatic.f90:70-138)
 * on the current device, in compact form: one flag byte per cell (its face
 * masks and maskT) and the metric factors as 2-D/1-D tables.  Applying it is
 * bit-identical to apply_op_3D with the reference's 27-entry cf. */
int32_t pyomgpu_nh_create(const pyomgpu_grid3d* grid, pyomgpu_nh** out);
void pyomgpu_nh_destroy(pyomgpu_nh* nh);
/* Device-side time limit of every grid-barrier wait (default 2 s). */
int32_t pyomgpu_nh_set_sync_timeout(pyomgpu_nh* nh, double seconds);
/* Failure-detection test hook, as pyomgpu_inject_barrier_stall. */
int32_t pyomgpu_nh_inject_barrier_stall(pyomgpu_nh* nh, int32_t enable);
/* Blocks of the CG launch (0 = one per brick, capped at the co-resident
 * maximum).  Reduction order follows the grid, so results change at rounding
 * level. */
int32_t pyomgpu_nh_set_grid(pyomgpu_nh* nh, int32_t blocks);
/* Brick shape of the CG sweeps: 32 x ty x kc cells staged with their halo in
 * shared memory (0, 0 = automatic: ty = min(8, ny), kc from a 26 KB box). */
int32_t pyomgpu_nh_set_brick(pyomgpu_nh* nh, int32_t ty, int32_t kc);
/* TMA pipeline depth of the CG sweeps: 2..4 stages (0 = automatic, 2). */
int32_t pyomgpu_nh_set_stages(pyomgpu_nh* nh, int32_t stages);
/* CG kernel: 1 = the grid-wide brick kernel, 2 = one thread-block cluster
 * (up to 16 blocks) with the fields resident in distributed shared memory
 * (grids of at most 110704 cells; cluster barriers instead of grid barriers,
 * so the barrier-stall hook does not apply), 0 = automatic (2 up to 32768
 * cells).  Reduction order differs, results change at rounding level. */
int32_t pyomgpu_nh_set_variant(pyomgpu_nh* nh, int32_t variant);
/* res = A p1 over the interior, zero halo (apply_op_3D).  (nx+4, ny+4, nz)
 * Fortran-layout arrays, host or device. */
int32_t pyomgpu_apply_op_3d(pyomgpu_nh* nh, const double* p1, double* res, pyomgpu_stream stream);
/* congrad_non_hydro (non_hydrostatic.f90:146-242): plain FP64 CG with
 * maskT-weighted dot_3D/absmax_3D, the reference's stopping estimate and
 * divergence test.  forc (read) and p = p_non_hydro(:,:,:,taup1) (in/out,
 * halo updated as the reference's whole-array update does) are Fortran-layout
 * (nx+4, ny+4, nz), host or device.  eps = congr_epsilon_non_hydro, max_it =
 * congr_max_itts_non_hydro; info->iterations = congr_itts_non_hydro.  An
 * immediate stop (zero initial residual) reports 0 iterations. */
int32_t pyomgpu_congrad_non_hydro(pyomgpu_nh* nh, const double* forc, double* p, double eps, int32_t max_it,
                                  pyomgpu_solve_info* info, pyomgpu_stream stream);

/* Model arrays of solve_non_hydrostatic (all DEVICE pointers, Fortran layout). */
typedef struct pyomgpu_state3d {
  int32_t taum1, tau, taup1;       /* 1-based time levels */
  int32_t itt;                     /* time step counter (itt == 0 copies p to tau and taum1) */
  int32_t congr_max_itts_non_hydro;
  int32_t congr_itts_non_hydro;    /* out */
  double dt_mom, AB_eps, congr_epsilon_non_hydro;
  double *u, *v, *w;               /* (nx+4, ny+4, nz, 3) */
  const double* dw;                /* (nx+4, ny+4, nz, 3) */
  const double* dw_mix;            /* (nx+4, ny+4, nz) */
  double* p_non_hydro;             /* (nx+4, ny+4, nz, 3) */
} pyomgpu_state3d;
/* solve_non_hydrostatic (non_hydrostatic.f90:5-63) on device-resident model
 * arrays: w(taup1) integrated, u/v/w(taup1) made cyclic, the divergence
 * forcing, the first guess 2 p(tau) - p(taum1), congrad_non_hydro, p made
 * cyclic (and copied to tau, taum1 when itt == 0), and the pressure-gradient
 * correction of u, v, w(taup1). */
int32_t pyomgpu_solve_non_hydrostatic(pyomgpu_nh* nh, pyomgpu_state3d* st, pyomgpu_solve_info* info,
                                      pyomgpu_stream stream);

/* ---- learned preconditioner (no counterpart in the reference) ----------------- */
/* Building block of the U-Net preconditioner: one 3x3 convolution (stride 1,
 * zero padding 1) on the tcgen05 tensor cores, BF16 operands, FP32
 * accumulation.  Activations are "channel-group planar" bf16:
 * [C/8][H][W][8] (a pixel's 8 channels of one group in 16 bytes).  All
 * pointers DEVICE.  w is f32 [cout][cin][3][3] (PyTorch order), bias f32
 * [cout] or NULL.  cin, cout in {16, 32, 64}.  epilogue:
 *   0  y = act(conv + bias (+ addend)) as planar bf16 [cout/8][H][W][8];
 *      gate (planar like y, may be NULL) zeroes y where gate <= 0 (the ReLU
 *      backward); pool_out (may be NULL; H, W even) receives the 2x2 average
 *      of y, planar [cout/8][H/2][W/2][8];
 *   1  y (2H x 2W) = act(conv broadcast to 2x2 blocks + addend) (decoder
 *      upsample + skip; addend required, 2H x 2W);
 *   2  y = f32 [H][W], channel 0 of conv + bias.
 * relu != 0 selects act = max(0, .).  flip != 0 runs the backward-data
 * convolution of a forward layer whose weight w is [cin][cout][3][3]
 * (channels transposed, kernel rotated 180 degrees). */
int32_t pyomgpu_conv3x3_bf16(int32_t cin, int32_t cout, int32_t H, int32_t W, const uint16_t* x, const float* w,
                             const float* bias, int32_t relu, int32_t epilogue, const uint16_t* gate,
                             const uint16_t* addend, void* y, uint16_t* pool_out, int32_t flip,
                             pyomgpu_stream stream);

/* The learned preconditioner of one grid: a 4-level U-Net (16/32/64/64
 * channels, 3x3 convolutions, BF16 weights and activations, FP32
 * accumulation) whose input is the residual scaled to unit rms, the unknown
 * mask, hur/mean(hur) and cosu, and whose output is a search direction
 * z ~ A^-1 r (scale free).  The context must have its islands set (Z).
 * training != 0 adds gradient and Adam buffers.  Parameters start at zero:
 * load them with pyomgpu_precond_set_params (f32, weights of the 12 layers in
 * PyTorch order [cout][cin][3][3], then their biases). */
typedef struct pyomgpu_precond pyomgpu_precond;
int64_t pyomgpu_precond_num_params(void);
int32_t pyomgpu_precond_create(pyomgpu_ctx* ctx, int32_t training, pyomgpu_precond** out);
void pyomgpu_precond_destroy(pyomgpu_precond* p);
/* Moves the network (parameters and optimiser state kept) to another grid of
 * the same size, e.g. to train on a family of grids. */
int32_t pyomgpu_precond_rebind(pyomgpu_precond* p, pyomgpu_ctx* ctx);
/* params: host or device, n = pyomgpu_precond_num_params(). */
int32_t pyomgpu_precond_set_params(pyomgpu_precond* p, const float* params, int64_t n);
int32_t pyomgpu_precond_get_params(pyomgpu_precond* p, float* params, int64_t n);
/* gradients of the last pyomgpu_precond_train_step / _unet_forward_backward */
int32_t pyomgpu_precond_get_grads(pyomgpu_precond* p, float* grads, int64_t n);
/* z = M(r); r, z Fortran-layout DEVICE arrays (z's halo holds the cyclic copies). */
int32_t pyomgpu_precond_apply(pyomgpu_precond* p, const double* r, double* z, pyomgpu_stream stream);
/* One training step on the pair (r, e): r a residual b - A x of the plain
 * solver, e = x* - x its error (Fortran-layout DEVICE arrays).  loss = 1 -
 * cos^2 of the angle between M(r) and e in the energy inner product
 * u^T D A v (D = dxu dyu cosu).  lr > 0 applies an Adam step (beta1 0.9,
 * beta2 0.999); lr = 0 only computes the gradients. */
int32_t pyomgpu_precond_train_step(pyomgpu_precond* p, const double* r, const double* e, float lr, float* loss,
                                   pyomgpu_stream stream);
/* The network alone, for gradient checks: x0 = planar bf16 input
 * [2][Hp][Wp][8] (Hp, Wp = ny, nx rounded up to multiples of 8), z = f32
 * output [Hp][Wp]; with gz (f32 [Hp][Wp], training only) also the parameter
 * gradients of sum(gz * z).  Host or device pointers. */
int32_t pyomgpu_unet_forward_backward(pyomgpu_precond* p, const uint16_t* x0, const float* gz, float* z,
                                      pyomgpu_stream stream);
/* Flexible CG (FCG(1)) preconditioned by the network, FP64 vectors and dot
 * products in the D-weighted inner product, to the FP64 true relative
 * residual rtol (as pyomgpu_solve_rtol).  When FCG stalls or breaks down the
 * iterate goes to the Jacobi-PCG kernel; the true residual decides.  info:
 * iterations (FCG + PCG), outer_iterations (1, or 2 when PCG took over),
 * rel_residual. */
int32_t pyomgpu_solve_fcg(pyomgpu_ctx* ctx, pyomgpu_precond* p, const double* forc, double* sol, double rtol,
                          int32_t max_iterations, pyomgpu_solve_info* info, pyomgpu_stream stream);

#ifdef __cplusplus
}
#endif
#endif
