/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY (see pyom_oracle.h).
 *
 * congrad_streamfunction as pyOM2's MPI build runs it on T processes,
 * restated with T POSIX threads over shared arrays.  It exists to time the
 * reference algorithm on every host core the machine gives (the CPU baseline
 * of the benchmark); the parity tests use the serial o_congrad_streamfunction.
 *
 * Decomposition: pe_decomposition (parallel_mpi.f90:11-44) with n_pes_i = 1,
 * n_pes_j = T: j_blk = (ny-1)/T + 1, thread t owns rows
 * js = t*j_blk + 1 .. je = min((t+1)*j_blk, ny) and every column.  Each thread
 * runs the serial routines (solve_streamfct.f90:153-422, solve_pressure.f90:
 * 254-274) over its own rows, in the reference's loop order.  The border
 * exchange (border_exchg_xy) becomes a barrier, since the neighbours' rows
 * live in the same arrays; setcyclic_xy (parallel_mpi.f90, n_pes_i = 1 case)
 * copies the cyclic columns of the thread's own rows.  global_sum / global_max
 * (parallel_mpi.f90:232-277, MPI_Allreduce) combine the T partial results in
 * thread order, so every thread obtains the same bits and takes the same
 * decisions.
 *
 * Rounding differs from the serial build only in the dot products and maxima
 * (partial sums per band), as between the reference's serial and MPI runs.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <sched.h>
#include <unistd.h>
#include <stdlib.h>
#include <string.h>

#include "pyom_oracle.h"

#define ONX 2
#define LDX(g) ((g)->nx + 2 * ONX)
#define LDY(g) ((g)->ny + 2 * ONX)
#define N2(g) ((size_t)LDX(g) * (size_t)LDY(g))
#define IX(g, i, j) ((size_t)((i) + ONX - 1) + (size_t)((j) + ONX - 1) * (size_t)LDX(g))
#define CF(g, cf, i, j, ii, jj) (cf)[IX(g, i, j) + (size_t)(((ii)-1) + ((jj)-1) * 3) * N2(g)]

static const double F_1EM10 = (double)1.e-10f; /* solve_streamfct.f90:262 */

#define PAD 8 /* doubles between two threads' partials (one cache line) */

typedef struct {
  double *part; /* T * PAD partials */
  int T;
  pthread_barrier_t bar;
} reduce_t;

static void barrier(reduce_t *r) { pthread_barrier_wait(&r->bar); }

/* global_sum: the partials of all threads in thread order */
static double all_sum(reduce_t *r, int t, double x) {
  r->part[t * PAD] = x;
  barrier(r);
  double s = r->part[0];
  for (int k = 1; k < r->T; k++) s = s + r->part[k * PAD];
  barrier(r);
  return s;
}

/* global_max */
static double all_max(reduce_t *r, int t, double x) {
  r->part[t * PAD] = x;
  barrier(r);
  double s = r->part[0];
  for (int k = 1; k < r->T; k++) s = r->part[k * PAD] > s ? r->part[k * PAD] : s;
  barrier(r);
  return s;
}

/* setcyclic_xy for rows js..je (the thread's own rows; cyclic x only, as
 * with n_pes_i = 1; a cyclic y domain is copied by the threads owning rows
 * 1..onx and ny-onx+1..ny after a barrier) */
static void cyclic_rows(const o_grid *g, double *p, int js, int je) {
  if (!g->cyclic_x) return;
  int nx = g->nx;
  for (int i = 1; i <= ONX; i++)
    for (int j = js; j <= je; j++) {
      p[IX(g, nx + i, j)] = p[IX(g, i, j)];
      p[IX(g, 1 - i, j)] = p[IX(g, nx - i + 1, j)];
    }
}
static void cyclic_y(const o_grid *g, double *p, int t, reduce_t *r) {
  if (!g->cyclic_y) return;
  barrier(r);
  if (t == 0) {
    int nx = g->nx, ny = g->ny;
    for (int j = 1; j <= ONX; j++)
      for (int i = 1 - ONX; i <= nx + ONX; i++) {
        p[IX(g, i, ny + j)] = p[IX(g, i, j)];
        p[IX(g, i, 1 - j)] = p[IX(g, i, ny - j + 1)];
      }
  }
}

/* apply_op (solve_pressure.f90:254-274) over rows js..je: the thread's rows
 * of res zeroed, then the 9 sweeps */
static void apply_op_rows(const o_grid *g, const double *cf, const double *p1, double *res, int js, int je) {
  for (int j = js; j <= je; j++) memset(&res[IX(g, 1 - ONX, j)], 0, (size_t)LDX(g) * sizeof(double));
  for (int jj = -1; jj <= 1; jj++)
    for (int ii = -1; ii <= 1; ii++)
      for (int j = js; j <= je; j++)
        for (int i = 1; i <= g->nx; i++)
          res[IX(g, i, j)] = res[IX(g, i, j)] + CF(g, cf, i, j, ii + 2, jj + 2) * p1[IX(g, i + ii, j + jj)];
}

static double dot_rows(const o_grid *g, const double *a, const double *b, int js, int je) {
  double s2 = 0;
  for (int j = js; j <= je; j++)
    for (int i = 1; i <= g->nx; i++) s2 = s2 + a[IX(g, i, j)] * b[IX(g, i, j)];
  return s2;
}

static double absmax_rows(const o_grid *g, const double *a, int js, int je) {
  double s2 = 0;
  for (int j = js; j <= je; j++)
    for (int i = 1; i <= g->nx; i++) {
      double v = fabs(a[IX(g, i, j)]);
      s2 = v > s2 ? v : s2;
    }
  return s2;
}

/* shared arguments and results of one threaded solve */
typedef struct {
  const o_grid *g;
  const double *cf, *forc;
  const o_islands *isl;
  double *sol, *res, *Z, *Zres, *ss, *As;
  double eps, rtol;
  int max_it, j_blk;
  reduce_t *red;
  int out_n, out_status, out_conv;
  double out_est;
} solve_t;

typedef struct {
  solve_t *S;
  int t;
} arg_t;

/* One process of the MPI build: rows js..je (solve_streamfct.f90:153-327). */
static void *solve_rows(void *vp) {
  arg_t *A = (arg_t *)vp;
  solve_t *S = A->S;
  const o_grid *g = S->g;
  const double *cf = S->cf, *forc = S->forc;
  double *sol = S->sol, *res = S->res, *Z = S->Z, *Zres = S->Zres, *ss = S->ss, *As = S->As;
  reduce_t *red = S->red;
  const double eps = S->eps, rtol = S->rtol;
  const int max_it = S->max_it;
  const int t = A->t;
  const int js = t * S->j_blk + 1, je = (t + 1) * S->j_blk < g->ny ? (t + 1) * S->j_blk : g->ny;
  const int nx = g->nx;
  double estimated_error = 0, zresmax, betakm1 = 0, betak, betak_min = 0, betaquot, s_dot_As, smax;
  double alpha, step, step1 = 0, convergence_rate, bnorm2 = 0;
  int n, status = 0, converged = 0;

  /* make_inv_sfc (:381-422) */
  for (int j = js; j <= je; j++)
    for (int i = 1; i <= nx; i++) Z[IX(g, i, j)] = CF(g, cf, i, j, 2, 2);
  for (int j = js; j <= je; j++)
    for (int i = 1; i <= nx; i++) Z[IX(g, i, j)] = Z[IX(g, i, j)] != 0.0 ? 1.0 / Z[IX(g, i, j)] : 0.0;
  barrier(red);
  if (t == 0 && S->isl) {
    const o_islands *isl = S->isl;
    for (int isle = 1; isle <= isl->nisle; isle++)
      for (int m = 1; m <= isl->nr_boundary[isle - 1]; m++) {
        size_t o = (size_t)(isle - 1) + (size_t)(m - 1) * isl->nisle;
        int i = isl->boundary[o], j = isl->boundary[o + (size_t)isl->nisle * isl->max_boundary];
        if (i >= 1 - ONX && i <= nx + ONX && j >= 1 - ONX && j <= g->ny + ONX) Z[IX(g, i, j)] = 0.0;
      }
  }
  /* sol's border exchange and cyclic copies (:191-192) */
  cyclic_rows(g, sol, js, je);
  cyclic_y(g, sol, t, red);
  barrier(red);
  apply_op_rows(g, cf, sol, res, js, je);
  for (int j = js; j <= je; j++)
    for (int i = 1; i <= nx; i++) res[IX(g, i, j)] = forc[IX(g, i, j)] - res[IX(g, i, j)];
  if (rtol > 0) {
    double b = 0;
    for (int j = js; j <= je; j++)
      for (int i = 1; i <= nx; i++)
        if (Z[IX(g, i, j)] != 0.0) b += forc[IX(g, i, j)] * forc[IX(g, i, j)];
    bnorm2 = all_sum(red, t, b);
  }
  n = 0;
  for (int j = js; j <= je; j++)
    for (int i = 1; i <= nx; i++) Zres[IX(g, i, j)] = Z[IX(g, i, j)] * res[IX(g, i, j)];
  zresmax = all_max(red, t, absmax_rows(g, Zres, js, je));
  if (100.0 * zresmax < eps) {
    estimated_error = 100.0 * zresmax;
    goto normal_end;
  }
  betakm1 = 1.0;
  for (n = 1; n <= max_it; n++) {
    for (int j = js; j <= je; j++)
      for (int i = 1; i <= nx; i++) Zres[IX(g, i, j)] = Z[IX(g, i, j)] * res[IX(g, i, j)];
    betak = all_sum(red, t, dot_rows(g, Zres, res, js, je));
    if (n == 1) {
      betak_min = fabs(betak);
    } else if (n > 2) {
      betak_min = betak_min < fabs(betak) ? betak_min : fabs(betak);
      if (fabs(betak) > 100.0 * betak_min) {
        status = 2;
        goto error_end;
      }
    }
    betaquot = betak / betakm1;
    for (int j = js; j <= je; j++)
      for (int i = 1; i <= nx; i++) ss[IX(g, i, j)] = Zres[IX(g, i, j)] + betaquot * ss[IX(g, i, j)];
    cyclic_rows(g, ss, js, je);
    cyclic_y(g, ss, t, red);
    barrier(red);
    apply_op_rows(g, cf, ss, As, js, je);
    s_dot_As = all_sum(red, t, dot_rows(g, ss, As, js, je));
    if (fabs(s_dot_As) < fabs(betak) * F_1EM10) {
      smax = all_max(red, t, absmax_rows(g, ss, js, je));
      estimated_error = 100.0 * smax;
      goto normal_end;
    }
    alpha = betak / s_dot_As;
    for (int j = js; j <= je; j++)
      for (int i = 1; i <= nx; i++) {
        sol[IX(g, i, j)] = sol[IX(g, i, j)] + alpha * ss[IX(g, i, j)];
        res[IX(g, i, j)] = res[IX(g, i, j)] - alpha * As[IX(g, i, j)];
      }
    smax = all_max(red, t, absmax_rows(g, ss, js, je));
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
      double rr = 0;
      for (int j = js; j <= je; j++)
        for (int i = 1; i <= nx; i++)
          if (Z[IX(g, i, j)] != 0.0) rr += res[IX(g, i, j)] * res[IX(g, i, j)];
      rr = all_sum(red, t, rr);
      if (bnorm2 > 0 ? (sqrt(rr / bnorm2) <= rtol) : (rr == 0.0)) {
        estimated_error = sqrt(rr);
        goto normal_end;
      }
    }
    betakm1 = betak;
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
  if (t == 0) {
    S->out_n = n;
    S->out_status = status;
    S->out_conv = converged;
    S->out_est = estimated_error;
  }
  return NULL;
}

/*
 * solve_streamfct.f90:153-327 on T threads (T <= 0: one per online CPU).
 * Same arguments, extension and status codes as the serial
 * o_congrad_streamfunction; the islands' Dirichlet points are set by the
 * serial make_inv_sfc loop over the perimeter lists, run by thread 0.
 */
int o_congrad_streamfunction_mt(const o_grid *g, const double *cf, const o_islands *isl, const double *forc,
                                double *sol, double eps, int max_it, double rtol, int nthreads, o_info *info) {
  size_t n2 = N2(g);
  int T = nthreads > 0 ? nthreads : o_max_threads();
  if (T > g->ny) T = g->ny;
  if (T > 1024) T = 1024;
  int j_blk = (g->ny - 1) / T + 1;
  /* pe_decomposition's check: the last block must not be empty */
  while (T > 1 && (T - 1) * j_blk + 1 > g->ny) {
    T--;
    j_blk = (g->ny - 1) / T + 1;
  }
  reduce_t red;
  red.T = T;
  red.part = (double *)calloc((size_t)T * PAD, sizeof(double));
  pthread_barrier_init(&red.bar, NULL, (unsigned)T);
  solve_t S = {g, cf, forc, isl, sol, NULL, NULL, NULL, NULL, NULL, eps, rtol, max_it, j_blk, &red, 0, 0, 0, 0.0};
  S.res = (double *)calloc(n2, sizeof(double));
  S.Z = (double *)calloc(n2, sizeof(double));
  S.Zres = (double *)calloc(n2, sizeof(double));
  S.ss = (double *)calloc(n2, sizeof(double));
  S.As = (double *)calloc(n2, sizeof(double));
  pthread_t *th = (pthread_t *)calloc((size_t)T, sizeof(pthread_t));
  arg_t *args = (arg_t *)calloc((size_t)T, sizeof(arg_t));
  for (int t = 0; t < T; t++) {
    args[t].S = &S;
    args[t].t = t;
    if (t > 0) pthread_create(&th[t], NULL, solve_rows, &args[t]);
  }
  solve_rows(&args[0]);
  for (int t = 1; t < T; t++) pthread_join(th[t], NULL);
  if (info) {
    info->iterations = S.out_n;
    info->converged = S.out_conv;
    info->status = S.out_status;
    info->estimated_error = S.out_est;
  }
  pthread_barrier_destroy(&red.bar);
  free(S.res);
  free(S.Z);
  free(S.Zres);
  free(S.ss);
  free(S.As);
  free(red.part);
  free(th);
  free(args);
  return S.out_status;
}

/* the host threads this process may run on */
int o_max_threads(void) {
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof set, &set) == 0) return CPU_COUNT(&set);
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}
