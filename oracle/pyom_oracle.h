/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C (FP64, sequential, reference loop order) restatement of pyOM2's
 * external-mode elliptic solve.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the product library never links
 * or calls it.
 *
 * Parity status: pinned to the reference's own source.  No Fortran compiler
 * exists in this image (none can be installed: no network, and the offline
 * wheelhouse carries no gfortran, flang or LFortran), and the reference ships
 * no tests or golden vectors for this path.  tests/golden/make_ref_golden.py
 * therefore runs pyOM2's Fortran routines (main_module, parallel_none,
 * numerics, island_module, streamfct_init, solve_streamfct, solve_pressure)
 * through the Fortran-subset translator oracle/f90sub.py and commits their
 * outputs; tests/test_oracle_vs_reference_source.py requires this restatement
 * to reproduce them bit for bit (grid metrics, masks, island lists, psin,
 * line_psin, CG iterates and iteration counts, solve_streamfunction and
 * solve_pressure steps), except where LAPACK's DGESV enters (scipy's LAPACK
 * there, the LU of o_dgesv here: rounding level).  Known-answer tests
 * (manufactured solutions, hand-checked island maps, operator identities)
 * and tests/golden/make_golden.py's fixtures remain as further checks.
 *
 * Layout: every 2-D array is Fortran-ordered with extents
 * (1-onx:nx+onx, 1-onx:ny+onx), onx = 2 (main_module.f90:35), i fastest.
 */
#ifndef PYOM_ORACLE_H
#define PYOM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct o_grid {
  int nx, ny;
  int cyclic_x, cyclic_y;
  const double *dxt, *dxu;                 /* [nx+4] */
  const double *dyt, *dyu, *cost, *cosu;   /* [ny+4] */
} o_grid;

typedef struct o_islands {
  int nisle, max_boundary;
  const int *boundary;    /* (nisle, max_boundary, 2) Fortran order */
  const int *line_dir;    /* (nisle, max_boundary, 2) */
  const int *nr_boundary; /* (nisle) */
} o_islands;

typedef struct o_info {
  int iterations;
  int converged;
  int status;              /* 0 ok, 1 max iterations, 2 diverged, 3 NaN */
  double estimated_error;
} o_info;

/* full model state for solve_streamfunction / solve_pressure */
typedef struct o_state {
  int nz;
  int taum1, tau, taup1;            /* 1-based time levels */
  int enable_free_surface;
  double dt_mom, AB_eps, grav, rho_0;
  double congr_epsilon;
  int congr_max_iterations;
  const double *dzt, *dzw;          /* [nz] */
  const double *hu, *hv, *hur, *hvr;
  const double *maskT, *maskU, *maskV;   /* (nx+4, ny+4, nz) */
  const double *rho;                /* (nx+4, ny+4, nz, 3) */
  double *u, *v, *du, *dv;          /* (nx+4, ny+4, nz, 3) */
  const double *du_mix, *dv_mix;    /* (nx+4, ny+4, nz) */
  double *p_hydro;                  /* (nx+4, ny+4, nz) */
  double *psi, *dpsi;               /* (nx+4, ny+4, 3) */
  const double *psin;               /* (nx+4, ny+4, nisle) */
  double *dpsin;                    /* (nisle, 3) */
  const double *line_psin;          /* (nisle, nisle) */
  int congr_itts;
  int status;
} o_state;

void o_setcyclic_xy(const o_grid *g, double *p);
void o_make_coeff_streamfunction(const o_grid *g, const double *hur, const double *hvr, double *cf);
void o_make_coeff_surf_press(const o_grid *g, const double *hu, const double *hv, const double *maskM,
                             int free_surface, double grav, double dt_mom, double *cf);
void o_apply_op(const o_grid *g, const double *cf, const double *p1, double *res);
void o_make_inv_sfc(const o_grid *g, const double *cf, const o_islands *isl, double *Z);
double o_dot_sfc(const o_grid *g, const double *p1, const double *p2);
double o_absmax_sfc(const o_grid *g, const double *p1);
double o_dot_sfp(const o_grid *g, const double *p1, const double *p2, const double *maskM);
double o_absmax_sfp(const o_grid *g, const double *p1, const double *maskM);

int o_congrad_streamfunction(const o_grid *g, const double *cf, const o_islands *isl, const double *forc,
                             double *sol, double eps, int max_it, double rtol, o_info *info);
int o_congrad_surf_press(const o_grid *g, const double *cf, const double *maskM, const double *forc,
                         double *psi, double eps, int max_it, double rtol, o_info *info);
/* o_congrad_streamfunction with cell-area-weighted inner products (exact
 * Jacobi-PCG on the symmetric S = D A; not in the reference) */
int o_congrad_streamfunction_w(const o_grid *g, const double *cf, const o_islands *isl, const double *forc,
                               double *sol, double eps, int max_it, double rtol, o_info *info);
/* congrad_streamfunction as the reference's MPI build runs it on nthreads
 * processes (pyom_oracle_mt.c; nthreads <= 0: one per CPU of the process) -- for
 * timing the reference algorithm on every host core */
int o_congrad_streamfunction_mt(const o_grid *g, const double *cf, const o_islands *isl, const double *forc,
                                double *sol, double eps, int max_it, double rtol, int nthreads, o_info *info);
int o_max_threads(void);

double o_rel_residual(const o_grid *g, const double *cf, const double *Z, const double *forc, const double *sol);

int o_isleperim(const int *kmt, int *map, int imt, int jmt, int cyclic, int mnisle, int maxipp, int maxq,
                int *nisle, int *nippts, int *iofs, int *iperm, int *jperm, int *nerror);
int o_island_map(const o_grid *g, const int *kbot, int mnisle, int maxipp, int maxq,
                 int *allmap, int *nisle, int *max_boundary);
int o_island_trace(const o_grid *g, const int *allmap, int nisle, int max_boundary, int mnisle, int maxipp,
                   int maxq, int *boundary, int *line_dir, int *nr_boundary);
double o_line_integral(const o_grid *g, const o_islands *isl, int isle, const double *uloc, const double *vloc,
                       int *err);
int o_psin_solve(const o_grid *g, const double *cf, const o_islands *isl, double eps, int max_it, double rtol,
                 int weighted, double *psin, int *iterations);
int o_line_psin(const o_grid *g, const o_islands *isl, const double *psin, const double *hur, const double *hvr,
                const double *maskU_top, const double *maskV_top, double *line_psin);
int o_dgesv(int n, double *a, int *ipiv, double *b);

/* ---- non-hydrostatic pressure (non_hydrostatic.f90) ---------------------------
 * 3-D arrays are (nx+4, ny+4, nz) Fortran order; cf is (nx+4, ny+4, nz, 3, 3, 3). */
typedef struct o_grid3 {
  o_grid g;
  int nz;
  const double *dzt, *dzw;                       /* [nz] */
  const double *maskT, *maskU, *maskV, *maskW;   /* (nx+4, ny+4, nz) */
} o_grid3;

void o_setcyclic_xyz(const o_grid3 *g, double *p);
void o_make_coeff_non_hydro(const o_grid3 *g, double *cf);
void o_apply_op_3d(const o_grid3 *g, const double *cf, const double *p1, double *res);
double o_dot_3d(const o_grid3 *g, const double *p1, const double *p2);
double o_absmax_3d(const o_grid3 *g, const double *p1);
int o_congrad_non_hydro(const o_grid3 *g, const double *cf, const double *forc, double *p, double eps, int max_it,
                        o_info *info);

/* model arrays of solve_non_hydrostatic (non_hydrostatic.f90:5-63) */
typedef struct o_state3 {
  int taum1, tau, taup1;            /* 1-based time levels */
  int itt;
  double dt_mom, AB_eps;
  double congr_epsilon_non_hydro;
  int congr_max_itts_non_hydro;
  double *u, *v, *w;                /* (nx+4, ny+4, nz, 3) */
  const double *dw;                 /* (nx+4, ny+4, nz, 3) */
  const double *dw_mix;             /* (nx+4, ny+4, nz) */
  double *p_non_hydro;              /* (nx+4, ny+4, nz, 3) */
  int congr_itts_non_hydro;         /* out */
  int status;                       /* out */
} o_state3;
int o_solve_non_hydrostatic(const o_grid3 *g, const double *cf, o_state3 *s);

int o_solve_streamfunction(const o_grid *g, const double *cf, const o_islands *isl, o_state *s);
int o_solve_pressure(const o_grid *g, const double *cf, o_state *s);

#ifdef __cplusplus
}
#endif
#endif
