/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY (see pyom_oracle.h).
 *
 * Plain C restatement of pyOM2's external-mode elliptic solve.  Each routine
 * names the reference lines it follows.  Loop order, the order of every
 * floating-point operation and the reference's control flow are kept, so the
 * results are those of the serial Fortran build compiled without FMA
 * contraction (the reference flags, site_specific.mk_x86_64-linux:8, do not
 * enable it; this file is compiled with -ffp-contract=off).
 *
 * Fortran default-real literals in the reference are float32 values; where
 * one enters a double expression it is written here as (double)<lit>f.
 */
#include "pyom_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ONX 2
#define LDX(g) ((g)->nx + 2 * ONX)
#define LDY(g) ((g)->ny + 2 * ONX)
#define N2(g) ((size_t)LDX(g) * (size_t)LDY(g))
/* Fortran (i,j), i in 1-onx..nx+onx, j in 1-onx..ny+onx */
#define IX(g, i, j) ((size_t)((i) + ONX - 1) + (size_t)((j) + ONX - 1) * (size_t)LDX(g))
#define X1(g, i) ((i) + ONX - 1) /* 1-D x arrays */
#define Y1(g, j) ((j) + ONX - 1) /* 1-D y arrays */
/* cf(i,j,ii,jj), ii,jj in 1..3 */
#define CF(g, cf, i, j, ii, jj) (cf)[IX(g, i, j) + (size_t)(((ii)-1) + ((jj)-1) * 3) * N2(g)]
/* boundary(isle,n,c) Fortran order (nisle, max_boundary, 2) */
#define BND(isl, a, isle, n, c) \
  (a)[(size_t)((isle)-1) + (size_t)((n)-1) * (isl)->nisle + (size_t)((c)-1) * (isl)->nisle * (isl)->max_boundary]

static const double F_1EM10 = (double)1.e-10f; /* solve_streamfct.f90:262 */

/* parallel_none.f90:188-211 */
void o_setcyclic_xy(const o_grid *g, double *p) {
  int nx = g->nx, ny = g->ny;
  if (g->cyclic_x) {
    for (int i = 1; i <= ONX; i++)
      for (int j = 1 - ONX; j <= ny + ONX; j++) {
        p[IX(g, nx + i, j)] = p[IX(g, i, j)];
        p[IX(g, 1 - i, j)] = p[IX(g, nx - i + 1, j)];
      }
  }
  if (g->cyclic_y) {
    for (int j = 1; j <= ONX; j++)
      for (int i = 1 - ONX; i <= nx + ONX; i++) {
        p[IX(g, i, ny + j)] = p[IX(g, i, j)];
        p[IX(g, i, 1 - j)] = p[IX(g, i, ny - j + 1)];
      }
  }
}

/* solve_streamfct.f90:123-148 */
void o_make_coeff_streamfunction(const o_grid *g, const double *hur, const double *hvr, double *cf) {
  memset(cf, 0, 9 * N2(g) * sizeof(double));
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) {
      double cu = g->cosu[Y1(g, j)];
      double cu2 = cu * cu;
      double a = hvr[IX(g, i + 1, j)] / g->dxu[X1(g, i)] / g->dxt[X1(g, i + 1)] / cu2;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - a;
      CF(g, cf, i, j, 3, 2) = CF(g, cf, i, j, 3, 2) + a;
      double b = hvr[IX(g, i, j)] / g->dxu[X1(g, i)] / g->dxt[X1(g, i)] / cu2;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - b;
      CF(g, cf, i, j, 1, 2) = CF(g, cf, i, j, 1, 2) + b;
      double c = hur[IX(g, i, j + 1)] / g->dyu[Y1(g, j)] / g->dyt[Y1(g, j + 1)] * g->cost[Y1(g, j + 1)] / cu;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - c;
      CF(g, cf, i, j, 2, 3) = CF(g, cf, i, j, 2, 3) + c;
      double d = hur[IX(g, i, j)] / g->dyu[Y1(g, j)] / g->dyt[Y1(g, j)] * g->cost[Y1(g, j)] / cu;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - d;
      CF(g, cf, i, j, 2, 1) = CF(g, cf, i, j, 2, 1) + d;
    }
}

/* solve_pressure.f90:87-131 */
void o_make_coeff_surf_press(const o_grid *g, const double *hu, const double *hv, const double *maskM,
                             int free_surface, double grav, double dt_mom, double *cf) {
  memset(cf, 0, 9 * N2(g) * sizeof(double));
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) {
      double ct = g->cost[Y1(g, j)];
      double ct2 = ct * ct;
      double mp = maskM[IX(g, i, j)] * maskM[IX(g, i + 1, j)];
      double mm = maskM[IX(g, i, j)] * maskM[IX(g, i - 1, j)];
      double a = mp * hu[IX(g, i, j)] / g->dxu[X1(g, i)] / g->dxt[X1(g, i)] / ct2;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - a;
      CF(g, cf, i, j, 3, 2) = CF(g, cf, i, j, 3, 2) + a;
      double b = mm * hu[IX(g, i - 1, j)] / g->dxu[X1(g, i - 1)] / g->dxt[X1(g, i)] / ct2;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - b;
      CF(g, cf, i, j, 1, 2) = CF(g, cf, i, j, 1, 2) + b;
      mp = maskM[IX(g, i, j)] * maskM[IX(g, i, j + 1)];
      mm = maskM[IX(g, i, j)] * maskM[IX(g, i, j - 1)];
      double c = mp * hv[IX(g, i, j)] / g->dyu[Y1(g, j)] / g->dyt[Y1(g, j)] * g->cosu[Y1(g, j)] / ct;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - c;
      CF(g, cf, i, j, 2, 3) = CF(g, cf, i, j, 2, 3) + c;
      double d = mm * hv[IX(g, i, j - 1)] / g->dyu[Y1(g, j - 1)] / g->dyt[Y1(g, j)] * g->cosu[Y1(g, j - 1)] / ct;
      CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - d;
      CF(g, cf, i, j, 2, 1) = CF(g, cf, i, j, 2, 1) + d;
    }
  if (free_surface) {
    double fs = 1.0 / (grav * (dt_mom * dt_mom));
    for (int j = 1; j <= g->ny; j++)
      for (int i = 1; i <= g->nx; i++)
        CF(g, cf, i, j, 2, 2) = CF(g, cf, i, j, 2, 2) - fs * maskM[IX(g, i, j)];
  }
}

/* solve_pressure.f90:254-274: 9 full sweeps, res zeroed first (halo included) */
void o_apply_op(const o_grid *g, const double *cf, const double *p1, double *res) {
  memset(res, 0, N2(g) * sizeof(double));
  for (int jj = -1; jj <= 1; jj++)
    for (int ii = -1; ii <= 1; ii++)
      for (int j = 1; j <= g->ny; j++)
        for (int i = 1; i <= g->nx; i++)
          res[IX(g, i, j)] = res[IX(g, i, j)] + CF(g, cf, i, j, ii + 2, jj + 2) * p1[IX(g, i + ii, j + jj)];
}

/* solve_streamfct.f90:381-422 */
void o_make_inv_sfc(const o_grid *g, const double *cf, const o_islands *isl, double *Z) {
  memset(Z, 0, N2(g) * sizeof(double));
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) Z[IX(g, i, j)] = CF(g, cf, i, j, 2, 2);
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) {
      if (Z[IX(g, i, j)] != 0.0)
        Z[IX(g, i, j)] = 1.0 / Z[IX(g, i, j)];
      else
        Z[IX(g, i, j)] = 0.0;
    }
  if (!isl) return;
  for (int isle = 1; isle <= isl->nisle; isle++)
    for (int n = 1; n <= isl->nr_boundary[isle - 1]; n++) {
      int i = BND(isl, isl->boundary, isle, n, 1);
      int j = BND(isl, isl->boundary, isle, n, 2);
      if (i >= 1 - ONX && i <= g->nx + ONX && j >= 1 - ONX && j <= g->ny + ONX) Z[IX(g, i, j)] = 0.0;
    }
}

/* solve_streamfct.f90:348-362 */
double o_dot_sfc(const o_grid *g, const double *p1, const double *p2) {
  double s2 = 0;
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) s2 = s2 + p1[IX(g, i, j)] * p2[IX(g, i, j)];
  return s2;
}

static inline double fmax_f(double a, double b) { return a > b ? a : b; }
static inline double fmin_f(double a, double b) { return a < b ? a : b; }

/* solve_streamfct.f90:331-345 */
double o_absmax_sfc(const o_grid *g, const double *p1) {
  double s2 = 0;
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) s2 = fmax_f(fabs(p1[IX(g, i, j)]), s2);
  return s2;
}

/* solve_pressure.f90:296-311 */
double o_dot_sfp(const o_grid *g, const double *p1, const double *p2, const double *maskM) {
  double s2 = 0;
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) s2 = s2 + p1[IX(g, i, j)] * p2[IX(g, i, j)] * maskM[IX(g, i, j)];
  return s2;
}

/* solve_pressure.f90:277-293 */
double o_absmax_sfp(const o_grid *g, const double *p1, const double *maskM) {
  double s2 = 0;
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) s2 = fmax_f(fabs(p1[IX(g, i, j)] * maskM[IX(g, i, j)]), s2);
  return s2;
}

/* ||b - A x||_2 / ||b||_2 over the points with Z != 0 (the unknowns). */
double o_rel_residual(const o_grid *g, const double *cf, const double *Z, const double *forc, const double *sol) {
  double *r = (double *)malloc(N2(g) * sizeof(double));
  double *s = (double *)malloc(N2(g) * sizeof(double));
  memcpy(s, sol, N2(g) * sizeof(double));
  o_setcyclic_xy(g, s); /* the caller's border exchange after the solve */
  o_apply_op(g, cf, s, r);
  free(s);
  double rr = 0, bb = 0;
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++) {
      if (Z[IX(g, i, j)] == 0.0) continue;
      double d = forc[IX(g, i, j)] - r[IX(g, i, j)];
      rr += d * d;
      bb += forc[IX(g, i, j)] * forc[IX(g, i, j)];
    }
  free(r);
  return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/* dot_sfc with every product weighted by the cell area dxu(i) dyu(j) cosu(j)
 * (the D of A = D^-1 S; not in the reference) */
static double dot_area(const o_grid *g, const double *p1, const double *p2) {
  double s2 = 0;
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++)
      s2 = s2 + (g->dxu[X1(g, i)] * (g->dyu[Y1(g, j)] * g->cosu[Y1(g, j)])) * p1[IX(g, i, j)] * p2[IX(g, i, j)];
  return s2;
}

static int congrad_core(const o_grid *g, const double *cf, const o_islands *isl, const double *forc, double *sol,
                        double eps, int max_it, double rtol, int weighted, o_info *info);

/*
 * solve_streamfct.f90:153-327 (congrad_streamfunction).
 * Extension for measurement only: rtol > 0 adds a stop on the recursively
 * updated residual, sqrt(sum_{Z!=0} res^2 / sum_{Z!=0} forc^2) <= rtol
 * (sum_{Z!=0} res_0^2 of the initial residual in place of the forcing's when
 * the forcing is zero; eps is then normally passed as 0 so the reference
 * criterion never fires).
 */
int o_congrad_streamfunction(const o_grid *g, const double *cf, const o_islands *isl, const double *forc,
                             double *sol, double eps, int max_it, double rtol, o_info *info) {
  return congrad_core(g, cf, isl, forc, sol, eps, max_it, rtol, 0, info);
}

/* The same with the inner products (beta, (s, As)) weighted by the cell area:
 * exact Jacobi-PCG on the symmetric S = D A (not in the reference). */
int o_congrad_streamfunction_w(const o_grid *g, const double *cf, const o_islands *isl, const double *forc,
                               double *sol, double eps, int max_it, double rtol, o_info *info) {
  return congrad_core(g, cf, isl, forc, sol, eps, max_it, rtol, 1, info);
}

static int congrad_core(const o_grid *g, const double *cf, const o_islands *isl, const double *forc, double *sol,
                        double eps, int max_it, double rtol, int weighted, o_info *info) {
  size_t n2 = N2(g);
  double *res = (double *)calloc(n2, sizeof(double));
  double *Z = (double *)calloc(n2, sizeof(double));
  double *Zres = (double *)calloc(n2, sizeof(double));
  double *ss = (double *)calloc(n2, sizeof(double));
  double *As = (double *)calloc(n2, sizeof(double));
  double estimated_error = 0, zresmax, betakm1 = 0, betak, betak_min = 0, betaquot, s_dot_As, smax;
  double alpha, step, step1 = 0, convergence_rate, bnorm2 = 0;
  int n, status = 0, converged = 0;
  int nx = g->nx, ny = g->ny;

  o_make_inv_sfc(g, cf, isl, Z);
  o_setcyclic_xy(g, sol);
  o_apply_op(g, cf, sol, res);
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) res[IX(g, i, j)] = forc[IX(g, i, j)] - res[IX(g, i, j)];
  if (rtol > 0) {
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++)
        if (Z[IX(g, i, j)] != 0.0) bnorm2 += forc[IX(g, i, j)] * forc[IX(g, i, j)];
    if (bnorm2 == 0.0)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
          if (Z[IX(g, i, j)] != 0.0) bnorm2 += res[IX(g, i, j)] * res[IX(g, i, j)];
  }
  n = 0;
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) Zres[IX(g, i, j)] = Z[IX(g, i, j)] * res[IX(g, i, j)];
  zresmax = o_absmax_sfc(g, Zres);
  if (100.0 * zresmax < eps) {
    estimated_error = 100.0 * zresmax;
    goto normal_end;
  }
  betakm1 = 1.0;
  for (n = 1; n <= max_it; n++) {
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) Zres[IX(g, i, j)] = Z[IX(g, i, j)] * res[IX(g, i, j)];
    betak = weighted ? dot_area(g, Zres, res) : o_dot_sfc(g, Zres, res);
    if (n == 1) {
      betak_min = fabs(betak);
    } else if (n > 2) {
      betak_min = fmin_f(betak_min, fabs(betak));
      if (fabs(betak) > 100.0 * betak_min) {
        status = 2;
        goto error_end;
      }
    }
    betaquot = betak / betakm1;
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) ss[IX(g, i, j)] = Zres[IX(g, i, j)] + betaquot * ss[IX(g, i, j)];
    o_setcyclic_xy(g, ss);
    o_apply_op(g, cf, ss, As);
    s_dot_As = weighted ? dot_area(g, ss, As) : o_dot_sfc(g, ss, As);
    if (fabs(s_dot_As) < fabs(betak) * F_1EM10) {
      smax = o_absmax_sfc(g, ss);
      estimated_error = 100.0 * smax;
      goto normal_end;
    }
    alpha = betak / s_dot_As;
    double rr = 0;
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        sol[IX(g, i, j)] = sol[IX(g, i, j)] + alpha * ss[IX(g, i, j)];
        res[IX(g, i, j)] = res[IX(g, i, j)] - alpha * As[IX(g, i, j)];
      }
    smax = o_absmax_sfc(g, ss);
    step = fabs(alpha) * smax;
    if (n == 1) {
      step1 = step;
      estimated_error = step;
      if (step < eps) goto normal_end;
    } else if (step < eps) {
      convergence_rate = exp(log(step / step1) / (double)(n - 1));
      estimated_error = step * convergence_rate / (1.0 - convergence_rate);
      if (estimated_error < eps) goto normal_end;
    }
    if (rtol > 0) {
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
          if (Z[IX(g, i, j)] != 0.0) rr += res[IX(g, i, j)] * res[IX(g, i, j)];
      if (bnorm2 > 0 ? (sqrt(rr / bnorm2) <= rtol) : (rr == 0.0)) {
        estimated_error = sqrt(rr);
        goto normal_end;
      }
    }
    betakm1 = betak;
  }
  status = 1; /* max iterations; n = max_it + 1 as after a completed DO loop */
  goto error_end;

normal_end:
  converged = 1;
  status = 0;
  goto done;
error_end:
  converged = 0;
  if (estimated_error != estimated_error) status = 3;
done:
  if (info) {
    info->iterations = n;
    info->converged = converged;
    info->status = status;
    info->estimated_error = estimated_error;
  }
  free(res);
  free(Z);
  free(Zres);
  free(ss);
  free(As);
  return status;
}

/*
 * solve_pressure.f90:137-249 (congrad_surf_press).  ``psi`` is psi(:,:,taup1),
 * updated over the full array including the halo as the reference does.
 * rtol > 0: extra stop on the masked residual norm (measurement only).
 */
int o_congrad_surf_press(const o_grid *g, const double *cf, const double *maskM, const double *forc,
                         double *psi, double eps, int max_it, double rtol, o_info *info) {
  size_t n2 = N2(g);
  double *res = (double *)calloc(n2, sizeof(double));
  double *p = (double *)calloc(n2, sizeof(double));
  double *Ap = (double *)calloc(n2, sizeof(double));
  double rsold, alpha, rsnew, fxa, step, step1 = 0, convergence_rate, estimated_error = 0, smax, rs_min = 0;
  double bnorm2 = 0;
  int n, status = 0, converged = 0;
  int nx = g->nx, ny = g->ny;

  o_apply_op(g, cf, psi, res);
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++) res[IX(g, i, j)] = forc[IX(g, i, j)] - res[IX(g, i, j)];
  memcpy(p, res, n2 * sizeof(double));
  o_setcyclic_xy(g, p);
  rsold = o_dot_sfp(g, res, res, maskM);
  if (rtol > 0) bnorm2 = o_dot_sfp(g, forc, forc, maskM);
  if (rsold == 0.0) {
    n = 0;
    goto normal_end;
  }
  for (n = 1; n <= max_it; n++) {
    o_apply_op(g, cf, p, Ap);
    fxa = o_dot_sfp(g, p, Ap, maskM);
    if (fxa == 0.0) goto normal_end;
    alpha = rsold / fxa;
    for (size_t k = 0; k < n2; k++) psi[k] = psi[k] + alpha * p[k];
    for (size_t k = 0; k < n2; k++) res[k] = res[k] - alpha * Ap[k];
    rsnew = o_dot_sfp(g, res, res, maskM);
    double bq = rsnew / rsold;
    for (size_t k = 0; k < n2; k++) p[k] = res[k] + bq * p[k];
    o_setcyclic_xy(g, p);
    rsold = rsnew;
    if (n == 1) {
      rs_min = fabs(rsnew);
    } else if (n > 2) {
      rs_min = fmin_f(rs_min, fabs(rsnew));
      if (fabs(rsnew) > 100.0 * rs_min) {
        status = 2;
        goto error_end;
      }
    }
    smax = o_absmax_sfp(g, p, maskM);
    step = fabs(alpha) * smax;
    if (n == 1) {
      step1 = step;
      estimated_error = step;
      if (step < eps) goto normal_end;
    } else if (step < eps) {
      convergence_rate = exp(log(step / step1) / (double)(n - 1));
      estimated_error = step * convergence_rate / (1.0 - convergence_rate);
      if (estimated_error < eps) goto normal_end;
    }
    if (estimated_error != estimated_error) {
      status = 3;
      goto error_end;
    }
    if (rtol > 0 && (bnorm2 > 0 ? sqrt(rsnew / bnorm2) <= rtol : rsnew == 0.0)) {
      estimated_error = sqrt(rsnew);
      goto normal_end;
    }
  }
  status = 1;
  goto error_end;
normal_end:
  converged = 1;
  status = 0;
  goto done;
error_end:
  converged = 0;
  if (estimated_error != estimated_error) status = 3;
done:
  if (info) {
    info->iterations = n;
    info->converged = converged;
    info->status = status;
    info->estimated_error = estimated_error;
  }
  free(res);
  free(p);
  free(Ap);
  return status;
}

/* ------------------------------------------------------------------------- */
/* island_module.f90:7-419                                                    */
/* ------------------------------------------------------------------------- */
typedef struct qstate {
  int *iq, *jq;
  int qfront, qback, maxq, maxqsize;
  int fault;
} qstate;

/* island_module.f90:276-288 */
static void qinit(qstate *q) {
  q->qfront = 1;
  q->qback = 0;
  q->iq[1] = 0;
  q->jq[1] = 0;
}
/* island_module.f90:291-317 */
static void qpush(qstate *q, int i, int j) {
  q->qback = q->qback + 1;
  if (q->qback > q->maxq) {
    if (q->qfront != 1) {
      int ishift = q->qfront - 1;
      for (int ip = q->qfront; ip <= q->qback - 1; ip++) {
        q->iq[ip - ishift] = q->iq[ip];
        q->jq[ip - ishift] = q->jq[ip];
      }
      q->qfront = 1;
      q->qback = q->qback - ishift;
    } else {
      q->fault = 1; /* 'queue fault in qpush' */
      q->qback = q->maxq;
      return;
    }
  }
  q->iq[q->qback] = i;
  q->jq[q->qback] = j;
  if (q->qback - q->qfront > q->maxqsize) q->maxqsize = q->qback - q->qfront;
}
/* island_module.f90:320-330 */
static void qpop(qstate *q, int *i, int *j) {
  *i = q->iq[q->qfront];
  *j = q->jq[q->qfront];
  q->qfront = q->qfront + 1;
}
static int qempty(const qstate *q) { return q->qfront > q->qback; }

/* island_module.f90:344-419 */
static int jn_isl(int j, int jmt) { return j < jmt ? j + 1 : -1; }
static int js_isl(int j) { return j > 1 ? j - 1 : -1; }
static int ie_isl(int i, int imt, int cyclic) {
  if (cyclic) return i < imt - 1 ? i + 1 : (i + 1) - imt + 2;
  return i < imt ? i + 1 : -1;
}
static int iw_isl(int i, int imt, int cyclic) {
  if (cyclic) return i > 2 ? i - 1 : (i - 1) + imt - 2;
  return i > 1 ? i - 1 : -1;
}

#define MAP(i, j) map[(size_t)((i)-1) + (size_t)((j)-1) * (size_t)imt]

/* island_module.f90:134-273; returns 0, or -1 (maxipp exceeded), -2 (queue fault) */
static int expand(int *map, int imt, int jmt, int cyclic, int label, qstate *q, int *nerror, int *iperm,
                  int *jperm, int *iofs, int *nippts, int maxipp) {
  for (;;) {
    if (q->fault) return -2;
    if (qempty(q)) {
      qinit(q);
      return 0;
    }
    int i, j;
    qpop(q, &i, &j);
    if (i == -1 || j == -1) continue;
    int m = MAP(i, j);
    if (m == label) continue;
    if (m == -label) continue;
    if (m == 1) {
      MAP(i, j) = label;
      int in_ = jn_isl(j, jmt), is_ = js_isl(j), ie = ie_isl(i, imt, cyclic), iw = iw_isl(i, imt, cyclic);
      qpush(q, i, in_);
      qpush(q, ie, in_);
      qpush(q, ie, j);
      qpush(q, ie, is_);
      qpush(q, i, is_);
      qpush(q, iw, is_);
      qpush(q, iw, j);
      qpush(q, iw, in_);
      continue;
    }
    if (m == 0 || m < 0) {
      if (m < 0) {
        *nerror = *nerror + 1; /* perimeter of another land mass: not relabelled */
        continue;
      }
      MAP(i, j) = -label;
      nippts[label] = nippts[label] + 1;
      if (iofs[label] + nippts[label] > maxipp) return -1;
      iperm[iofs[label] + nippts[label]] = i;
      jperm[iofs[label] + nippts[label]] = j;
      continue;
    }
    *nerror = *nerror + 1; /* labelled for another land mass */
  }
}

/*
 * island_module.f90:7-127.  kmt/map are (imt,jmt) Fortran order, 1-based.
 * nippts/iofs need mnisle+1 entries, iperm/jperm maxipp+1 (1-based use).
 * Returns 0; -1 maxipp too small; -2 queue fault; -3 mnisle too small.
 */
int o_isleperim(const int *kmt, int *map, int imt, int jmt, int cyclic, int mnisle, int maxipp, int maxq,
                int *nisle, int *nippts, int *iofs, int *iperm, int *jperm, int *nerror_out) {
  const int land = 1, ocean = 0;
  for (int i = 1; i <= imt; i++)
    for (int j = 1; j <= jmt; j++) MAP(i, j) = kmt[(size_t)(i - 1) + (size_t)(j - 1) * imt] > 0 ? ocean : land;
  qstate q;
  q.maxq = maxq;
  q.iq = (int *)calloc((size_t)maxq + 2, sizeof(int));
  q.jq = (int *)calloc((size_t)maxq + 2, sizeof(int));
  q.maxqsize = 0;
  q.fault = 0;
  qinit(&q);
  int label = 2, nerror = 0, rc = 0;
  iofs[label] = 0;
  nippts[label] = 0;
  int jnorth = jmt, iwest, ieast;
  if (cyclic) {
    iwest = 2;
    ieast = imt - 1;
  } else {
    iwest = 1;
    ieast = imt;
  }
  for (int j = jnorth; j >= 1; j--)
    for (int i = iwest; i <= ieast; i++) {
      if (MAP(i, j) == land) {
        qpush(&q, i, j);
        rc = expand(map, imt, jmt, cyclic, label, &q, &nerror, iperm, jperm, iofs, nippts, maxipp);
        if (rc) goto out;
        label = label + 1;
        if (label > mnisle) {
          rc = -3;
          goto out;
        }
        iofs[label] = iofs[label - 1] + nippts[label - 1];
        nippts[label] = 0;
      }
    }
  *nisle = label - 1;
  for (int i = iwest; i <= ieast; i++)
    for (int j = 1; j <= jnorth; j++)
      if (MAP(i, j) != 0) MAP(i, j) = MAP(i, j) - (MAP(i, j) > 0 ? 1 : -1);
  for (int isle = 2; isle <= *nisle; isle++) {
    iofs[isle - 1] = iofs[isle];
    nippts[isle - 1] = nippts[isle];
  }
  *nisle = *nisle - 1;
  if (cyclic)
    for (int j = 1; j <= jmt; j++) {
      MAP(1, j) = MAP(imt - 1, j);
      MAP(imt, j) = MAP(2, j);
    }
out:
  if (nerror_out) *nerror_out = nerror;
  free(q.iq);
  free(q.jq);
  return rc;
}
#undef MAP

/*
 * streamfct_init.f90:35-87: global land map, first isleperim over all land
 * masses, cyclic halo copy, paranoia check, max_boundary.  allmap has the
 * 2-D halo layout.  Returns 0 or a negative error.
 */
int o_island_map(const o_grid *g, const int *kbot, int mnisle, int maxipp, int maxq, int *allmap, int *nisle,
                 int *max_boundary) {
  int nx = g->nx, ny = g->ny;
  size_t n2 = N2(g);
  int *kmt = (int *)calloc(n2, sizeof(int));
  int *nippts = (int *)calloc((size_t)mnisle + 2, sizeof(int));
  int *iofs = (int *)calloc((size_t)mnisle + 2, sizeof(int));
  int *iperm = (int *)calloc((size_t)maxipp + 2, sizeof(int));
  int *jperm = (int *)calloc((size_t)maxipp + 2, sizeof(int));
  int rc, nerr;
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      if (kbot[IX(g, i, j)] > 0) kmt[IX(g, i, j)] = 5;
  if (g->cyclic_x)
    for (int i = 1; i <= ONX; i++)
      for (int j = 1 - ONX; j <= ny + ONX; j++) {
        kmt[IX(g, nx + i, j)] = kmt[IX(g, i, j)];
        kmt[IX(g, 1 - i, j)] = kmt[IX(g, nx - i + 1, j)];
      }
  rc = o_isleperim(kmt, allmap, LDX(g), LDY(g), g->cyclic_x, mnisle, maxipp, maxq, nisle, nippts, iofs, iperm,
                   jperm, &nerr);
  if (rc) goto out;
  if (g->cyclic_x)
    for (int i = 1; i <= ONX; i++)
      for (int j = 1 - ONX; j <= ny + ONX; j++) {
        allmap[IX(g, nx + i, j)] = allmap[IX(g, i, j)];
        allmap[IX(g, 1 - i, j)] = allmap[IX(g, nx - i + 1, j)];
      }
  /* paranoia check, streamfct_init.f90:64-83 */
  for (int isle = 1; isle <= *nisle; isle++) {
    int found = 0;
    for (size_t k = 0; k < n2 && !found; k++) found = allmap[k] == isle;
    if (!found) {
      rc = -5;
      goto out;
    }
  }
  {
    int mx = 0;
    for (int isle = 1; isle <= *nisle; isle++)
      if (nippts[isle] > mx) mx = nippts[isle];
    *max_boundary = 20 * mx;
  }
out:
  free(kmt);
  free(nippts);
  free(iofs);
  free(iperm);
  free(jperm);
  return rc;
}

/*
 * streamfct_init.f90:95-267: per island, re-run isleperim on that island
 * alone, find a start point and walk the perimeter with the right-hand rule.
 * Returns 0; -6 no starting point; -7 lost track; -8 max_boundary exceeded;
 * -9 map index out of range; other negatives from isleperim.
 */
int o_island_trace(const o_grid *g, const int *allmap, int nisle, int max_boundary, int mnisle, int maxipp,
                   int maxq, int *boundary, int *line_dir, int *nr_boundary) {
  int nx = g->nx, ny = g->ny;
  size_t n2 = N2(g);
  int *kmt = (int *)malloc(n2 * sizeof(int));
  int *map = (int *)calloc(n2, sizeof(int));
  int *nippts = (int *)calloc((size_t)mnisle + 2, sizeof(int));
  int *iofs = (int *)calloc((size_t)mnisle + 2, sizeof(int));
  int *iperm = (int *)calloc((size_t)maxipp + 2, sizeof(int));
  int *jperm = (int *)calloc((size_t)maxipp + 2, sizeof(int));
  o_islands I = {nisle, max_boundary, boundary, line_dir, nr_boundary};
  const o_islands *isl = &I;
  int rc = 0;
  memset(boundary, 0, sizeof(int) * (size_t)nisle * max_boundary * 2);
  memset(line_dir, 0, sizeof(int) * (size_t)nisle * max_boundary * 2);
  memset(nr_boundary, 0, sizeof(int) * (size_t)nisle);
#define M(i, j) map[IX(g, i, j)]
#define INB(i, j) ((i) >= 1 - ONX && (i) <= nx + ONX && (j) >= 1 - ONX && (j) <= ny + ONX)
#define SETB(arr, n, a, b)                            \
  do {                                                \
    ((int *)(arr))[(size_t)(isle - 1) + (size_t)((n)-1) * nisle] = (a); \
    ((int *)(arr))[(size_t)(isle - 1) + (size_t)((n)-1) * nisle + (size_t)nisle * max_boundary] = (b); \
  } while (0)
  for (int isle = 1; isle <= nisle; isle++) {
    int ni, nerr;
    for (size_t k = 0; k < n2; k++) kmt[k] = allmap[k] == isle ? 0 : 1;
    rc = o_isleperim(kmt, map, LDX(g), LDY(g), g->cyclic_x, mnisle, maxipp, maxq, &ni, nippts, iofs, iperm,
                     jperm, &nerr);
    if (rc) goto out;
    int n = 1, cont = 0, ij[2] = {0, 0}, dir[2] = {0, 0};
    for (int i = nx / 2 + 1; i <= nx && !cont; i++)
      for (int j = 0; j <= ny; j++) {
        if (M(i, j) == 1 && M(i, j + 1) == -1) {
          ij[0] = i; ij[1] = j; cont = 1;
          dir[0] = 1; dir[1] = 0;
          SETB(boundary, n, ij[0] - 1, ij[1]);
          break;
        }
        if (M(i, j) == -1 && M(i, j + 1) == 1) {
          ij[0] = i - 1; ij[1] = j; cont = 1;
          dir[0] = -1; dir[1] = 0;
          SETB(boundary, n, ij[0] + 1, ij[1]);
          break;
        }
      }
    if (!cont) {
      for (int i = nx / 2; i >= 1 && !cont; i--)
        for (int j = 0; j <= ny; j++) {
          if (M(i, j) == 1 && M(i, j + 1) == -1) {
            ij[0] = i; ij[1] = j; cont = 1;
            dir[0] = 1; dir[1] = 0;
            SETB(boundary, n, ij[0] - 1, ij[1]);
            break;
          }
          if (M(i, j) == -1 && M(i, j + 1) == 1) {
            ij[0] = i - 1; ij[1] = j; cont = 1;
            dir[0] = -1; dir[1] = 0;
            SETB(boundary, n, ij[0] + 1, ij[1]);
            break;
          }
        }
      if (!cont) {
        rc = -6;
        goto out;
      }
    }
    SETB(line_dir, n, dir[0], dir[1]);
    n = 2;
    if (n > max_boundary) {
      rc = -8;
      goto out;
    }
    SETB(boundary, n, ij[0], ij[1]);
    cont = 1;
    while (cont) {
      int ijp[2] = {0, 0}, ijr[2] = {0, 0};
      if (dir[0] == 0 && dir[1] == 1) { ijp[0] = ij[0]; ijp[1] = ij[1] + 1; ijr[0] = ij[0] + 1; ijr[1] = ij[1] + 1; }
      if (dir[0] == -1 && dir[1] == 0) { ijp[0] = ij[0]; ijp[1] = ij[1]; ijr[0] = ij[0]; ijr[1] = ij[1] + 1; }
      if (dir[0] == 0 && dir[1] == -1) { ijp[0] = ij[0] + 1; ijp[1] = ij[1]; ijr[0] = ij[0]; ijr[1] = ij[1]; }
      if (dir[0] == 1 && dir[1] == 0) { ijp[0] = ij[0] + 1; ijp[1] = ij[1] + 1; ijr[0] = ij[0] + 1; ijr[1] = ij[1]; }
      if (!INB(ijp[0], ijp[1]) || !INB(ijr[0], ijr[1])) {
        rc = -9;
        goto out;
      }
      int a = M(ijp[0], ijp[1]), b = M(ijr[0], ijr[1]);
      if (a == -1 && b == 1) {
        /* go forward */
      } else if (a == -1 && b == -1) {
        int d0 = dir[1], d1 = -dir[0];
        dir[0] = d0; dir[1] = d1;
      } else if (a == 1 && b == 1) {
        int d0 = -dir[1], d1 = dir[0];
        dir[0] = d0; dir[1] = d1;
      } else if (a == 1 && b == -1) {
        int d0 = -dir[1], d1 = dir[0];
        dir[0] = d0; dir[1] = d1;
      } else {
        rc = -7;
        goto out;
      }
      SETB(line_dir, n, dir[0], dir[1]);
      ij[0] += dir[0];
      ij[1] += dir[1];
      if (BND(isl, boundary, isle, 1, 1) == ij[0] && BND(isl, boundary, isle, 1, 2) == ij[1]) cont = 0;
      if (g->cyclic_x && dir[0] == 1 && dir[1] == 0 && ij[0] > nx) ij[0] = ij[0] - nx;
      if (g->cyclic_x && dir[0] == -1 && dir[1] == 0 && ij[0] < 1) ij[0] = ij[0] + nx;
      if (BND(isl, boundary, isle, 1, 1) == ij[0] && BND(isl, boundary, isle, 1, 2) == ij[1]) cont = 0;
      if (cont) {
        n = n + 1;
        if (n > max_boundary) {
          rc = -8;
          goto out;
        }
        SETB(boundary, n, ij[0], ij[1]);
      }
    }
    nr_boundary[isle - 1] = n;
  }
#undef M
#undef INB
#undef SETB
out:
  free(kmt);
  free(map);
  free(nippts);
  free(iofs);
  free(iperm);
  free(jperm);
  return rc;
}

/* streamfct_init.f90:311-377 (serial: is=js=0 because is_pe=js_pe=1) */
double o_line_integral(const o_grid *g, const o_islands *isl, int isle, const double *uloc, const double *vloc,
                       int *err) {
  double line = 0;
  int is = 0, js = 0, ie = g->nx, je = g->ny;
  if (err) *err = 0;
  for (int n = 1; n <= isl->nr_boundary[isle - 1]; n++) {
    int i = BND(isl, isl->boundary, isle, n, 1);
    int j = BND(isl, isl->boundary, isle, n, 2);
    if (i >= is && i <= ie && j >= js && j <= je) {
      int d0 = BND(isl, isl->line_dir, isle, n, 1);
      int d1 = BND(isl, isl->line_dir, isle, n, 2);
      if (d0 == 1 && d1 == 0) {
        line = line + vloc[IX(g, i, j)] * g->dyu[Y1(g, j)] + uloc[IX(g, i, j + 1)] * g->dxu[X1(g, i)] * g->cost[Y1(g, j + 1)];
      } else if (d0 == -1 && d1 == 0) {
        line = line - vloc[IX(g, i + 1, j)] * g->dyu[Y1(g, j)] - uloc[IX(g, i, j)] * g->dxu[X1(g, i)] * g->cost[Y1(g, j)];
      } else if (d0 == 0 && d1 == 1) {
        line = line + vloc[IX(g, i, j)] * g->dyu[Y1(g, j)] - uloc[IX(g, i, j)] * g->dxu[X1(g, i)] * g->cost[Y1(g, j)];
      } else if (d0 == 0 && d1 == -1) {
        line = line + uloc[IX(g, i, j + 1)] * g->dxu[X1(g, i)] * g->cost[Y1(g, j + 1)] - vloc[IX(g, i + 1, j)] * g->dyu[Y1(g, j)];
      } else {
        if (err) *err = -10; /* 'missing line_dir in line integral' */
      }
    }
  }
  return line;
}

/* streamfct_init.f90:272-287: one CG solve per island with forc = 0 and
 * psin = 1 on the island's own perimeter.  psin is (nx+4, ny+4, nisle). */
int o_psin_solve(const o_grid *g, const double *cf, const o_islands *isl, double eps, int max_it, double rtol,
                 int weighted, double *psin, int *iterations) {
  size_t n2 = N2(g);
  double *forc = (double *)calloc(n2, sizeof(double));
  int worst = 0;
  for (int isle = 1; isle <= isl->nisle; isle++) {
    double *p = psin + (size_t)(isle - 1) * n2;
    memset(p, 0, n2 * sizeof(double));
    for (int n = 1; n <= isl->nr_boundary[isle - 1]; n++) {
      int i = BND(isl, isl->boundary, isle, n, 1);
      int j = BND(isl, isl->boundary, isle, n, 2);
      if (i >= 1 - ONX && i <= g->nx + ONX && j >= 1 - ONX && j <= g->ny + ONX) p[IX(g, i, j)] = 1.0;
    }
    o_setcyclic_xy(g, p);
    o_info info;
    int st = congrad_core(g, cf, isl, forc, p, eps, max_it, rtol, weighted, &info);
    if (iterations) iterations[isle - 1] = info.iterations;
    if (st > worst) worst = st;
    o_setcyclic_xy(g, p);
  }
  free(forc);
  return worst;
}

/* velocity of a streamfunction field as in streamfct_init.f90:295-300 and
 * solve_streamfct.f90:68-74 */
static void psi_velocity(const o_grid *g, const double *p, const double *hur, const double *hvr,
                         const double *maskU_top, const double *maskV_top, double *fpx, double *fpy) {
  size_t n2 = N2(g);
  memset(fpx, 0, n2 * sizeof(double));
  memset(fpy, 0, n2 * sizeof(double));
  for (int j = 1 - ONX + 1; j <= g->ny + ONX; j++)
    for (int i = 1 - ONX + 1; i <= g->nx + ONX; i++) {
      fpx[IX(g, i, j)] = -maskU_top[IX(g, i, j)] * (p[IX(g, i, j)] - p[IX(g, i, j - 1)]) / g->dyt[Y1(g, j)] * hur[IX(g, i, j)];
      fpy[IX(g, i, j)] = maskV_top[IX(g, i, j)] * (p[IX(g, i, j)] - p[IX(g, i - 1, j)]) /
                         (g->cosu[Y1(g, j)] * g->dxt[X1(g, i)]) * hvr[IX(g, i, j)];
    }
}

/* streamfct_init.f90:292-303 */
int o_line_psin(const o_grid *g, const o_islands *isl, const double *psin, const double *hur, const double *hvr,
                const double *maskU_top, const double *maskV_top, double *line_psin) {
  size_t n2 = N2(g);
  double *fpx = (double *)malloc(n2 * sizeof(double));
  double *fpy = (double *)malloc(n2 * sizeof(double));
  int nisle = isl->nisle, err = 0, e;
  for (int n = 1; n <= nisle; n++)
    for (int isle = 1; isle <= nisle; isle++) {
      psi_velocity(g, psin + (size_t)(isle - 1) * n2, hur, hvr, maskU_top, maskV_top, fpx, fpy);
      line_psin[(size_t)(n - 1) + (size_t)(isle - 1) * nisle] = o_line_integral(g, isl, n, fpx, fpy, &e);
      if (e) err = e;
    }
  free(fpx);
  free(fpy);
  return err;
}

/* LAPACK DGESV semantics (DGETF2 partial pivoting + DGETRS), column-major
 * a(n,n), one right-hand side.  Returns info (0 ok, k>0: U(k,k) == 0). */
int o_dgesv(int n, double *a, int *ipiv, double *b) {
  int info = 0;
  const double sfmin = 2.2250738585072014e-308;
#define A(i, j) a[(size_t)(i) + (size_t)(j) * n]
  for (int k = 0; k < n; k++) {
    int p = k;
    double mx = fabs(A(k, k));
    for (int i = k + 1; i < n; i++)
      if (fabs(A(i, k)) > mx) {
        mx = fabs(A(i, k));
        p = i;
      }
    ipiv[k] = p + 1;
    if (A(p, k) != 0.0) {
      if (p != k)
        for (int j = 0; j < n; j++) {
          double t = A(k, j);
          A(k, j) = A(p, j);
          A(p, j) = t;
        }
      if (fabs(A(k, k)) >= sfmin) {
        double r = 1.0 / A(k, k);
        for (int i = k + 1; i < n; i++) A(i, k) = A(i, k) * r;
      } else {
        for (int i = k + 1; i < n; i++) A(i, k) = A(i, k) / A(k, k);
      }
    } else if (info == 0) {
      info = k + 1;
    }
    for (int j = k + 1; j < n; j++) {
      double t = A(k, j);
      if (t != 0.0)
        for (int i = k + 1; i < n; i++) A(i, j) = A(i, j) - A(i, k) * t;
    }
  }
  if (info) return info;
  for (int k = 0; k < n; k++) {
    int p = ipiv[k] - 1;
    if (p != k) {
      double t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
  for (int j = 0; j < n; j++)
    for (int i = j + 1; i < n; i++) b[i] = b[i] - A(i, j) * b[j];
  for (int j = n - 1; j >= 0; j--) {
    b[j] = b[j] / A(j, j);
    for (int i = 0; i < j; i++) b[i] = b[i] - A(i, j) * b[j];
  }
#undef A
  return 0;
}

/* 3-D helpers: (nx+4, ny+4, nz[, 3]) Fortran order */
#define I3(g, i, j, k) (IX(g, i, j) + (size_t)((k)-1) * N2(g))
#define I4(g, nz, i, j, k, t) (I3(g, i, j, k) + (size_t)((t)-1) * (size_t)(nz) * N2(g))

static void hydrostatic_and_gradient(const o_grid *g, o_state *s) {
  int nz = s->nz, tau = s->tau;
  size_t n2 = N2(g);
  double fxa = s->grav / s->rho_0;
  /* solve_streamfct.f90:25-29 / solve_pressure.f90:20-24 */
  for (size_t q = 0; q < n2; q++)
    s->p_hydro[q + (size_t)(nz - 1) * n2] =
        0.5 * s->rho[q + (size_t)(nz - 1) * n2 + (size_t)(tau - 1) * nz * n2] * fxa * s->dzw[nz - 1] *
        s->maskT[q + (size_t)(nz - 1) * n2];
  for (int k = nz - 1; k >= 1; k--)
    for (size_t q = 0; q < n2; q++) {
      size_t o = q + (size_t)(k - 1) * n2, o1 = q + (size_t)k * n2, t = (size_t)(tau - 1) * nz * n2;
      s->p_hydro[o] = s->maskT[o] * (s->p_hydro[o1] + 0.5 * (s->rho[o1 + t] + s->rho[o + t]) * fxa * s->dzw[k - 1]);
    }
  /* solve_streamfct.f90:32-37 */
  for (int j = 1; j <= g->ny; j++)
    for (int i = 1; i <= g->nx; i++)
      for (int k = 1; k <= nz; k++) {
        size_t d = I4(g, nz, i, j, k, tau);
        s->du[d] = s->du[d] - (s->p_hydro[I3(g, i + 1, j, k)] - s->p_hydro[I3(g, i, j, k)]) /
                                  (g->dxu[X1(g, i)] * g->cost[Y1(g, j)]) * s->maskU[I3(g, i, j, k)];
        s->dv[d] = s->dv[d] - (s->p_hydro[I3(g, i, j + 1, k)] - s->p_hydro[I3(g, i, j, k)]) / g->dyu[Y1(g, j)] *
                                  s->maskV[I3(g, i, j, k)];
      }
}

/* solve_streamfct.f90:10-120 */
int o_solve_streamfunction(const o_grid *g, const double *cf, const o_islands *isl, o_state *s) {
  int nx = g->nx, ny = g->ny, nz = s->nz;
  int tau = s->tau, taum1 = s->taum1, taup1 = s->taup1;
  size_t n2 = N2(g);
  double *fpx = (double *)calloc(n2, sizeof(double));
  double *fpy = (double *)calloc(n2, sizeof(double));
  double *forc = (double *)calloc(n2, sizeof(double));
  int nisle = isl ? isl->nisle : 0, rc = 0;
  double AB = s->AB_eps, dt = s->dt_mom;

  hydrostatic_and_gradient(g, s);
  /* :39-44 */
  for (int k = 1; k <= nz; k++)
    for (size_t q = 0; q < n2; q++) {
      size_t o = q + (size_t)(k - 1) * n2, t = (size_t)(tau - 1) * nz * n2;
      fpx[q] = fpx[q] + (s->du[o + t] + s->du_mix[o]) * s->maskU[o] * s->dzt[k - 1];
      fpy[q] = fpy[q] + (s->dv[o + t] + s->dv_mix[o]) * s->maskV[o] * s->dzt[k - 1];
    }
  for (size_t q = 0; q < n2; q++) {
    fpx[q] = fpx[q] * s->hur[q];
    fpy[q] = fpy[q] * s->hvr[q];
  }
  o_setcyclic_xy(g, fpx);
  o_setcyclic_xy(g, fpy);
  /* :49-53 */
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      forc[IX(g, i, j)] = (fpy[IX(g, i + 1, j)] - fpy[IX(g, i, j)]) / (g->cosu[Y1(g, j)] * g->dxu[X1(g, i)]) -
                          (g->cost[Y1(g, j + 1)] * fpx[IX(g, i, j + 1)] - g->cost[Y1(g, j)] * fpx[IX(g, i, j)]) /
                              (g->cosu[Y1(g, j)] * g->dyu[Y1(g, j)]);
  /* :56-59 */
  double *dp1 = s->dpsi + (size_t)(taup1 - 1) * n2;
  double *dp0 = s->dpsi + (size_t)(tau - 1) * n2;
  double *dpm = s->dpsi + (size_t)(taum1 - 1) * n2;
  for (size_t q = 0; q < n2; q++) dp1[q] = 2 * dp0[q] - dpm[q];
  o_info info;
  int st = o_congrad_streamfunction(g, cf, isl, forc, dp1, s->congr_epsilon, s->congr_max_iterations, 0.0, &info);
  s->congr_itts = info.iterations;
  s->status = st;
  o_setcyclic_xy(g, dp1);
  /* :61-88 */
  if (nisle > 1) {
    double *line_forc = (double *)calloc((size_t)nisle, sizeof(double));
    double *line_psi0 = (double *)calloc((size_t)nisle, sizeof(double));
    double *aloc = (double *)calloc((size_t)nisle * nisle, sizeof(double));
    int *ipiv = (int *)calloc((size_t)nisle, sizeof(int));
    int e;
    for (int k = 2; k <= nisle; k++) line_forc[k - 1] = o_line_integral(g, isl, k, fpx, fpy, &e);
    for (int k = 2; k <= nisle; k++) {
      memset(fpx, 0, n2 * sizeof(double));
      memset(fpy, 0, n2 * sizeof(double));
      const double *mU = s->maskU + (size_t)(nz - 1) * n2, *mV = s->maskV + (size_t)(nz - 1) * n2;
      for (int j = 1 - ONX + 1; j <= ny + ONX; j++)
        for (int i = 1 - ONX + 1; i <= nx + ONX; i++) {
          fpx[IX(g, i, j)] = -mU[IX(g, i, j)] * (dp1[IX(g, i, j)] - dp1[IX(g, i, j - 1)]) / g->dyt[Y1(g, j)] *
                             s->hur[IX(g, i, j)];
          fpy[IX(g, i, j)] = mV[IX(g, i, j)] * (dp1[IX(g, i, j)] - dp1[IX(g, i - 1, j)]) /
                             (g->cosu[Y1(g, j)] * g->dxt[X1(g, i)]) * s->hvr[IX(g, i, j)];
        }
      line_psi0[k - 1] = o_line_integral(g, isl, k, fpx, fpy, &e);
    }
    for (int k = 0; k < nisle; k++) line_forc[k] = line_forc[k] - line_psi0[k];
    int m = nisle - 1;
    for (int c = 0; c < m; c++)
      for (int r = 0; r < m; r++) aloc[(size_t)r + (size_t)c * m] = s->line_psin[(size_t)(r + 1) + (size_t)(c + 1) * nisle];
    int info2 = o_dgesv(m, aloc, ipiv, line_forc + 1);
    if (info2 != 0) rc = 5;
    for (int k = 2; k <= nisle; k++) s->dpsin[(size_t)(k - 1) + (size_t)(tau - 1) * nisle] = line_forc[k - 1];
    free(line_forc);
    free(line_psi0);
    free(aloc);
    free(ipiv);
  }
  /* :91-96 */
  double *ps1 = s->psi + (size_t)(taup1 - 1) * n2, *ps0 = s->psi + (size_t)(tau - 1) * n2;
  for (size_t q = 0; q < n2; q++) ps1[q] = ps0[q] + dt * ((1.5 + AB) * dp1[q] - (0.5 + AB) * dp0[q]);
  for (int isle = 2; isle <= nisle; isle++) {
    double c = dt * ((1.5 + AB) * s->dpsin[(size_t)(isle - 1) + (size_t)(tau - 1) * nisle] -
                     (0.5 + AB) * s->dpsin[(size_t)(isle - 1) + (size_t)(taum1 - 1) * nisle]);
    const double *pn = s->psin + (size_t)(isle - 1) * n2;
    for (size_t q = 0; q < n2; q++) ps1[q] = ps1[q] + c * pn[q];
  }
  size_t n3 = n2 * (size_t)nz;
  for (size_t q = 0; q < n3; q++) {
    size_t a1 = q + (size_t)(taup1 - 1) * n3, a0 = q + (size_t)(tau - 1) * n3, am = q + (size_t)(taum1 - 1) * n3;
    s->u[a1] = s->u[a0] + dt * (s->du_mix[q] + (1.5 + AB) * s->du[a0] - (0.5 + AB) * s->du[am]) * s->maskU[q];
    s->v[a1] = s->v[a0] + dt * (s->dv_mix[q] + (1.5 + AB) * s->dv[a0] - (0.5 + AB) * s->dv[am]) * s->maskV[q];
  }
  /* :99 set_obc_streamfct: no open boundaries in this build (no-op) */
  /* :102-110 */
  memset(fpx, 0, n2 * sizeof(double));
  memset(fpy, 0, n2 * sizeof(double));
  for (int k = 1; k <= nz; k++)
    for (size_t q = 0; q < n2; q++) {
      size_t o = q + (size_t)(k - 1) * n2, a1 = o + (size_t)(taup1 - 1) * n3;
      fpx[q] = fpx[q] + s->u[a1] * s->maskU[o] * s->dzt[k - 1];
      fpy[q] = fpy[q] + s->v[a1] * s->maskV[o] * s->dzt[k - 1];
    }
  for (int k = 1; k <= nz; k++)
    for (size_t q = 0; q < n2; q++) {
      size_t o = q + (size_t)(k - 1) * n2, a1 = o + (size_t)(taup1 - 1) * n3;
      s->u[a1] = s->u[a1] - fpx[q] * s->maskU[o] * s->hur[q];
      s->v[a1] = s->v[a1] - fpy[q] * s->maskV[o] * s->hvr[q];
    }
  /* :113-118 */
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      for (int k = 1; k <= nz; k++) {
        size_t a1 = I4(g, nz, i, j, k, taup1);
        s->u[a1] = s->u[a1] - s->maskU[I3(g, i, j, k)] * (ps1[IX(g, i, j)] - ps1[IX(g, i, j - 1)]) / g->dyt[Y1(g, j)] *
                                  s->hur[IX(g, i, j)];
        s->v[a1] = s->v[a1] + s->maskV[I3(g, i, j, k)] * (ps1[IX(g, i, j)] - ps1[IX(g, i - 1, j)]) /
                                  (g->cosu[Y1(g, j)] * g->dxt[X1(g, i)]) * s->hvr[IX(g, i, j)];
      }
  free(fpx);
  free(fpy);
  free(forc);
  return rc ? rc : st;
}

/* solve_pressure.f90:10-82 */
int o_solve_pressure(const o_grid *g, const double *cf, o_state *s) {
  int nx = g->nx, ny = g->ny, nz = s->nz;
  int tau = s->tau, taum1 = s->taum1, taup1 = s->taup1;
  size_t n2 = N2(g), n3 = n2 * (size_t)nz;
  double *fpx = (double *)calloc(n2, sizeof(double));
  double *fpy = (double *)calloc(n2, sizeof(double));
  double *forc = (double *)calloc(n2, sizeof(double));
  double AB = s->AB_eps, dt = s->dt_mom;
  const double *maskM = s->maskT + (size_t)(nz - 1) * n2;

  hydrostatic_and_gradient(g, s);
  for (size_t q = 0; q < n3; q++) {
    size_t a1 = q + (size_t)(taup1 - 1) * n3, a0 = q + (size_t)(tau - 1) * n3, am = q + (size_t)(taum1 - 1) * n3;
    s->u[a1] = s->u[a0] + dt * (s->du_mix[q] + (1.5 + AB) * s->du[a0] - (0.5 + AB) * s->du[am]) * s->maskU[q];
    s->v[a1] = s->v[a0] + dt * (s->dv_mix[q] + (1.5 + AB) * s->dv[a0] - (0.5 + AB) * s->dv[am]) * s->maskV[q];
  }
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t o = I3(g, i, j, k), a1 = o + (size_t)(taup1 - 1) * n3;
        fpx[IX(g, i, j)] = fpx[IX(g, i, j)] + s->u[a1] * s->maskU[o] * s->dzt[k - 1] / dt;
        fpy[IX(g, i, j)] = fpy[IX(g, i, j)] + s->v[a1] * s->maskV[o] * s->dzt[k - 1] / dt;
      }
  o_setcyclic_xy(g, fpx);
  o_setcyclic_xy(g, fpy);
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      forc[IX(g, i, j)] = (fpx[IX(g, i, j)] - fpx[IX(g, i - 1, j)]) / (g->cost[Y1(g, j)] * g->dxt[X1(g, i)]) +
                          (g->cosu[Y1(g, j)] * fpy[IX(g, i, j)] - g->cosu[Y1(g, j - 1)] * fpy[IX(g, i, j - 1)]) /
                              (g->cost[Y1(g, j)] * g->dyt[Y1(g, j)]);
  double *ps1 = s->psi + (size_t)(taup1 - 1) * n2, *ps0 = s->psi + (size_t)(tau - 1) * n2,
         *psm = s->psi + (size_t)(taum1 - 1) * n2;
  if (s->enable_free_surface)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++)
        forc[IX(g, i, j)] = forc[IX(g, i, j)] - ps0[IX(g, i, j)] / (s->grav * (dt * dt)) * maskM[IX(g, i, j)];
  for (size_t q = 0; q < n2; q++) ps1[q] = 2 * ps0[q] - psm[q];
  o_info info;
  int st = o_congrad_surf_press(g, cf, maskM, forc, ps1, s->congr_epsilon, s->congr_max_iterations, 0.0, &info);
  s->congr_itts = info.iterations;
  s->status = st;
  o_setcyclic_xy(g, ps1);
  for (int j = 1; j <= ny; j++)
    for (int i = 1; i <= nx; i++)
      for (int k = 1; k <= nz; k++) {
        size_t a1 = I4(g, nz, i, j, k, taup1);
        s->u[a1] = s->u[a1] - dt * (ps1[IX(g, i + 1, j)] - ps1[IX(g, i, j)]) / (g->dxu[X1(g, i)] * g->cost[Y1(g, j)]) *
                                  s->maskU[I3(g, i, j, k)];
        s->v[a1] = s->v[a1] - dt * (ps1[IX(g, i, j + 1)] - ps1[IX(g, i, j)]) / g->dyu[Y1(g, j)] * s->maskV[I3(g, i, j, k)];
      }
  free(fpx);
  free(fpy);
  free(forc);
  return st;
}

/* ------------------------------------------------------------------------- */
/* non_hydrostatic.f90: make_coeff_non_hydro, apply_op_3D, dot_3D,            */
/* absmax_3D, congrad_non_hydro                                               */
/* ------------------------------------------------------------------------- */
#define N3(g3) (N2(&(g3)->g) * (size_t)(g3)->nz)
#define IX3(g3, i, j, k) (IX(&(g3)->g, i, j) + (size_t)((k)-1) * N2(&(g3)->g))
#define CF3(g3, cf, i, j, k, ii, jj, kk) \
  (cf)[IX3(g3, i, j, k) + (size_t)(((ii)-1) + 3 * (((jj)-1) + 3 * ((kk)-1))) * N3(g3)]

/* setcyclic_xyz (parallel_none.f90): setcyclic_xy on every level */
void o_setcyclic_xyz(const o_grid3 *g3, double *p) {
  for (int k = 1; k <= g3->nz; k++) o_setcyclic_xy(&g3->g, p + (size_t)(k - 1) * N2(&g3->g));
}

/* non_hydrostatic.f90:70-138, same accumulation order */
void o_make_coeff_non_hydro(const o_grid3 *g3, double *cf) {
  const o_grid *g = &g3->g;
  const int nx = g->nx, ny = g->ny, nz = g3->nz;
  memset(cf, 0, N3(g3) * 27 * sizeof(double));
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        const double c2 = g->cost[Y1(g, j)] * g->cost[Y1(g, j)];
        double mp = g3->maskU[IX3(g3, i, j, k)], mm = g3->maskU[IX3(g3, i - 1, j, k)];
        CF3(g3, cf, i, j, k, 2, 2, 2) -= mp / g->dxu[X1(g, i)] / g->dxt[X1(g, i)] / c2;
        CF3(g3, cf, i, j, k, 3, 2, 2) += mp / g->dxu[X1(g, i)] / g->dxt[X1(g, i)] / c2;
        CF3(g3, cf, i, j, k, 2, 2, 2) -= mm / g->dxu[X1(g, i - 1)] / g->dxt[X1(g, i)] / c2;
        CF3(g3, cf, i, j, k, 1, 2, 2) += mm / g->dxu[X1(g, i - 1)] / g->dxt[X1(g, i)] / c2;
        mp = g3->maskV[IX3(g3, i, j, k)];
        mm = g3->maskV[IX3(g3, i, j - 1, k)];
        CF3(g3, cf, i, j, k, 2, 2, 2) -= mp / g->dyu[Y1(g, j)] / g->dyt[Y1(g, j)] * g->cosu[Y1(g, j)] / g->cost[Y1(g, j)];
        CF3(g3, cf, i, j, k, 2, 3, 2) += mp / g->dyu[Y1(g, j)] / g->dyt[Y1(g, j)] * g->cosu[Y1(g, j)] / g->cost[Y1(g, j)];
        CF3(g3, cf, i, j, k, 2, 2, 2) -=
            mm / g->dyu[Y1(g, j - 1)] / g->dyt[Y1(g, j)] * g->cosu[Y1(g, j - 1)] / g->cost[Y1(g, j)];
        CF3(g3, cf, i, j, k, 2, 1, 2) +=
            mm / g->dyu[Y1(g, j - 1)] / g->dyt[Y1(g, j)] * g->cosu[Y1(g, j - 1)] / g->cost[Y1(g, j)];
      }
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        if (k < nz) { /* k = 1 and 2..nz-1: the upper face */
          const double mp = g3->maskW[IX3(g3, i, j, k)];
          CF3(g3, cf, i, j, k, 2, 2, 2) -= mp / g3->dzw[k - 1] / g3->dzt[k - 1];
          CF3(g3, cf, i, j, k, 2, 2, 3) += mp / g3->dzw[k - 1] / g3->dzt[k - 1];
        }
        if (k > 1) { /* 2..nz-1 and nz: the lower face */
          const double mm = g3->maskW[IX3(g3, i, j, k - 1)];
          CF3(g3, cf, i, j, k, 2, 2, 2) -= mm / g3->dzw[k - 2] / g3->dzt[k - 1];
          CF3(g3, cf, i, j, k, 2, 2, 1) += mm / g3->dzw[k - 2] / g3->dzt[k - 1];
        }
      }
}

/* non_hydrostatic.f90:247-276: res = 0, then sum over (kk, jj, ii) outermost */
void o_apply_op_3d(const o_grid3 *g3, const double *cf, const double *p1, double *res) {
  const o_grid *g = &g3->g;
  const int nz = g3->nz;
  memset(res, 0, N3(g3) * sizeof(double));
  for (int kk = -1; kk <= 1; kk++)
    for (int jj = -1; jj <= 1; jj++)
      for (int ii = -1; ii <= 1; ii++)
        for (int k = 1; k <= nz; k++) {
          const int kpkk = k + kk < 1 ? 1 : (k + kk > nz ? nz : k + kk);
          for (int j = 1; j <= g->ny; j++)
            for (int i = 1; i <= g->nx; i++)
              res[IX3(g3, i, j, k)] =
                  res[IX3(g3, i, j, k)] + CF3(g3, cf, i, j, k, ii + 2, jj + 2, kk + 2) * p1[IX3(g3, i + ii, j + jj, kpkk)];
        }
}

/* non_hydrostatic.f90:300-322 */
double o_dot_3d(const o_grid3 *g3, const double *p1, const double *p2) {
  double s2 = 0;
  for (int k = 1; k <= g3->nz; k++)
    for (int j = 1; j <= g3->g.ny; j++)
      for (int i = 1; i <= g3->g.nx; i++) {
        const size_t q = IX3(g3, i, j, k);
        s2 = s2 + p1[q] * p2[q] * g3->maskT[q];
      }
  return s2;
}

/* non_hydrostatic.f90:279-297 */
double o_absmax_3d(const o_grid3 *g3, const double *p1) {
  double s2 = 0;
  for (int k = 1; k <= g3->nz; k++)
    for (int j = 1; j <= g3->g.ny; j++)
      for (int i = 1; i <= g3->g.nx; i++) {
        const size_t q = IX3(g3, i, j, k);
        s2 = fmax_f(fabs(p1[q] * g3->maskT[q]), s2);
      }
  return s2;
}

/* non_hydrostatic.f90:146-242; p is p_non_hydro(:,:,:,taup1), in/out.  An
 * immediate stop (rsold == 0) reports 0 iterations (the reference leaves n
 * undefined there). */
int o_congrad_non_hydro(const o_grid3 *g3, const double *cf, const double *forc, double *p_nh, double eps, int max_it,
                        o_info *info) {
  const size_t n3 = N3(g3);
  double *res = (double *)calloc(n3, sizeof(double));
  double *p = (double *)calloc(n3, sizeof(double));
  double *Ap = (double *)calloc(n3, sizeof(double));
  double rsold, alpha, rsnew, fxa, step, step1 = 0, convergence_rate, estimated_error = 0, smax, rs_min = 0;
  int n, status = 0, converged = 0;

  o_apply_op_3d(g3, cf, p_nh, res);
  for (int k = 1; k <= g3->nz; k++)
    for (int j = 1; j <= g3->g.ny; j++)
      for (int i = 1; i <= g3->g.nx; i++) res[IX3(g3, i, j, k)] = forc[IX3(g3, i, j, k)] - res[IX3(g3, i, j, k)];
  memcpy(p, res, n3 * sizeof(double));
  o_setcyclic_xyz(g3, p);
  rsold = o_dot_3d(g3, res, res);
  if (rsold == 0.0) {
    n = 0;
    goto normal_end;
  }
  for (n = 1; n <= max_it; n++) {
    o_apply_op_3d(g3, cf, p, Ap);
    fxa = o_dot_3d(g3, p, Ap);
    if (fxa == 0.0) goto normal_end;
    alpha = rsold / fxa;
    for (size_t q = 0; q < n3; q++) p_nh[q] = p_nh[q] + alpha * p[q];
    for (size_t q = 0; q < n3; q++) res[q] = res[q] - alpha * Ap[q];
    rsnew = o_dot_3d(g3, res, res);
    const double bq = rsnew / rsold;
    for (size_t q = 0; q < n3; q++) p[q] = res[q] + bq * p[q];
    o_setcyclic_xyz(g3, p);
    rsold = rsnew;
    if (n == 1) {
      rs_min = fabs(rsnew);
    } else if (n > 2) {
      rs_min = fmin_f(rs_min, fabs(rsnew));
      if (fabs(rsnew) > 100.0 * rs_min) {
        status = 2;
        goto error_end;
      }
    }
    smax = o_absmax_3d(g3, p);
    step = fabs(alpha) * smax;
    if (n == 1) {
      step1 = step;
      estimated_error = step;
      if (step < eps) goto normal_end;
    } else if (step < eps) {
      convergence_rate = exp(log(step / step1) / (double)(n - 1));
      estimated_error = step * convergence_rate / (1.0 - convergence_rate);
      if (estimated_error < eps) goto normal_end;
    }
  }
  status = 1;
  goto error_end;
normal_end:
  converged = 1;
  status = 0;
  goto done;
error_end:
  converged = 0;
  if (estimated_error != estimated_error) status = 3;
done:
  if (info) {
    info->iterations = n;
    info->converged = converged;
    info->status = status;
    info->estimated_error = estimated_error;
  }
  free(res);
  free(p);
  free(Ap);
  return status;
}

/* non_hydrostatic.f90:5-63.  forc's halo is never read by the solve (the
 * reference leaves it uninitialised); it is zero here. */
int o_solve_non_hydrostatic(const o_grid3 *g3, const double *cf, o_state3 *s) {
  const o_grid *g = &g3->g;
  const int nx = g->nx, ny = g->ny, nz = g3->nz;
  const size_t n3 = N3(g3);
  const int X = nx + 4, Y = ny + 4;
  double *u = s->u + (size_t)(s->taup1 - 1) * n3;
  double *v = s->v + (size_t)(s->taup1 - 1) * n3;
  double *w = s->w + (size_t)(s->taup1 - 1) * n3;
  const double *w_tau = s->w + (size_t)(s->tau - 1) * n3;
  const double *dw_tau = s->dw + (size_t)(s->tau - 1) * n3;
  const double *dw_taum1 = s->dw + (size_t)(s->taum1 - 1) * n3;
  double *p1 = s->p_non_hydro + (size_t)(s->taup1 - 1) * n3;
  double *p0 = s->p_non_hydro + (size_t)(s->tau - 1) * n3;
  double *pm = s->p_non_hydro + (size_t)(s->taum1 - 1) * n3;
  /* :13-15 integrate w forward (whole levels k < nz) */
  for (int k = 1; k < nz; k++)
    for (int jj = 0; jj < Y; jj++)
      for (int ii = 0; ii < X; ii++) {
        const size_t q = (size_t)ii + (size_t)X * ((size_t)jj + (size_t)Y * (size_t)(k - 1));
        w[q] = w_tau[q] + s->dt_mom *
                              (s->dw_mix[q] + (1.5 + s->AB_eps) * dw_tau[q] - (0.5 + s->AB_eps) * dw_taum1[q]) *
                              g3->maskW[q];
      }
  /* :19-24 */
  o_setcyclic_xyz(g3, u);
  o_setcyclic_xyz(g3, v);
  o_setcyclic_xyz(g3, w);
  /* :25-36 */
  double *forc = (double *)calloc(n3, sizeof(double));
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        const double cj = g->cost[Y1(g, j)];
        forc[IX3(g3, i, j, k)] = (u[IX3(g3, i, j, k)] - u[IX3(g3, i - 1, j, k)]) / (cj * g->dxt[X1(g, i)]) +
                                 (g->cosu[Y1(g, j)] * v[IX3(g3, i, j, k)] -
                                  g->cosu[Y1(g, j - 1)] * v[IX3(g3, i, j - 1, k)]) /
                                     (cj * g->dyt[Y1(g, j)]);
      }
  for (size_t q = 0; q < N2(g); q++) forc[q] = forc[q] + w[q] / g3->dzt[0];
  for (int k = 2; k <= nz; k++) {
    const size_t o = (size_t)(k - 1) * N2(g), om = (size_t)(k - 2) * N2(g);
    for (size_t q = 0; q < N2(g); q++) forc[o + q] = forc[o + q] + (w[o + q] - w[om + q]) / g3->dzt[k - 1];
  }
  for (size_t q = 0; q < n3; q++) forc[q] = forc[q] / s->dt_mom;
  /* :40-48 */
  for (size_t q = 0; q < n3; q++) p1[q] = 2 * p0[q] - pm[q];
  o_info info;
  s->status = o_congrad_non_hydro(g3, cf, forc, p1, s->congr_epsilon_non_hydro, s->congr_max_itts_non_hydro, &info);
  s->congr_itts_non_hydro = info.iterations;
  free(forc);
  o_setcyclic_xyz(g3, p1);
  if (s->itt == 0) {
    memcpy(p0, p1, n3 * sizeof(double));
    memcpy(pm, p1, n3 * sizeof(double));
  }
  /* :52-61 */
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        const size_t q = IX3(g3, i, j, k);
        u[q] = u[q] - s->dt_mom * (p1[IX3(g3, i + 1, j, k)] - p1[q]) / (g->dxu[X1(g, i)] * g->cost[Y1(g, j)]) *
                          g3->maskU[q];
        v[q] = v[q] - s->dt_mom * (p1[IX3(g3, i, j + 1, k)] - p1[q]) / g->dyu[Y1(g, j)] * g3->maskV[q];
      }
  for (int k = 1; k < nz; k++) {
    const size_t o = (size_t)(k - 1) * N2(g), op = (size_t)k * N2(g);
    for (size_t q = 0; q < N2(g); q++)
      w[o + q] = w[o + q] - s->dt_mom * (p1[op + q] - p1[o + q]) / g3->dzw[k - 1] * g3->maskW[o + q];
  }
  return s->status;
}
