// Momentum tendencies of pyOM2's time step on the GPU (momentum.f90:4-152
// with the parts its hydrostatic configurations without turbulence closures
// use): Coriolis and metric terms, surface wind stress, momentum advection
// (momentum_advection.f90:1-76), implicit vertical friction with a given
// viscosity kappaM (vertical_friction.f90:109-226), harmonic lateral friction
// (harmonic_friction.f90:4-124) and linear bottom friction
// (bottom_friction.f90:48-135), plus vertical_velocity (vertical_velocity.f90).
//
// Every kernel evaluates the reference's expressions term by term in the
// reference's order, and this file is compiled without FMA contraction
// (build.py), so the tendencies equal the serial Fortran build's bit for bit
// on the interior points.  One thread owns one water column (i, j) and walks
// k, recomputing the fluxes across its own faces (the reference stores them in
// module arrays; recomputing gives the same values).  The energy-dissipation
// diagnostics the reference accumulates on the side (K_diss_*, calc_diss) feed
// closures outside this path and are not formed.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/pyomgpu.h"
#include "common.cuh"

namespace pyomgpu {
void set_last_error(const char* msg);  // capi.cu
// grid size and the 1-D device metrics of a context (capi.cu)
int ctx_grid1d(pyomgpu_ctx* c, int* nx, int* ny, const double** out6, int* cyclic_x, int* cyclic_y);

namespace {

int mfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}

// Fortran layout: (i, j) in (-1 .. nx+2, -1 .. ny+2), k in 1 .. nz, time level t in 1 .. 3
struct MG {
  int nx, ny, nz;
  size_t n2;
  __device__ __forceinline__ size_t ij(int i, int j) const { return (size_t)(i + 1) + (size_t)(j + 1) * (nx + 4); }
  __device__ __forceinline__ size_t k3(int i, int j, int k) const { return ij(i, j) + (size_t)(k - 1) * n2; }
  __device__ __forceinline__ size_t k4(int i, int j, int k, int t) const {
    return k3(i, j, k) + (size_t)(t - 1) * n2 * nz;
  }
};

struct MomDev {
  MG g;
  int tau, taup1, coord_degree;
  int hor_friction, cos_scaling, cos_power, bottom_friction, implicit_vert;
  double dt_mom, A_h, r_bot;
  // 1-D: x and y arrays at Fortran index + 1, z arrays at k - 1
  const double *dxt, *dxu, *dyt, *dyu, *cost, *cosu, *tantr, *dzt, *dzw;
  const double *maskU, *maskV, *maskW, *kappaM;
  const int* kbot;
  const double *coriolis_t, *area_t, *area_u, *area_v, *taux, *tauy;
  double *u, *v, *w, *du, *dv, *du_mix, *dv_mix;
};

// x**n for an integer n >= 0 as the reference evaluates it (a product of n
// factors; cos powers of 1 to 3 occur)
__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  if (n >= 1) r = x;
  for (int k = 2; k <= n; k++) r = r * x;
  return r;
}

// ---- Coriolis, metric terms, wind stress, advection -> du, dv(tau) ---------------
// momentum.f90:11-35 (du_cor, dv_cor), :82-93 (du = du_cor, stress), :95-97 (+ du_adv);
// momentum_advection.f90:13-76.
__global__ void k_mom_cor_adv(MomDev m) {
  const MG& g = m.g;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nx * g.ny) return;
  const int i = 1 + t % g.nx, j = 1 + t / g.nx;
  const int tau = m.tau, nz = g.nz;
  const double* ut = m.u + (size_t)(tau - 1) * g.n2 * nz;
  const double* vt = m.v + (size_t)(tau - 1) * g.n2 * nz;
  const double* wt = m.w + (size_t)(tau - 1) * g.n2 * nz;
  const double dxt_i = m.dxt[i + 1], dxt_ip = m.dxt[i + 2], dxu_i = m.dxu[i + 1];
  const double dyt_j = m.dyt[j + 1], dyt_jp = m.dyt[j + 2], dyu_j = m.dyu[j + 1];
  const double cost_j = m.cost[j + 1], cost_jp = m.cost[j + 2], cosu_j = m.cosu[j + 1];
  const double area_u = m.area_u[g.ij(i, j)], area_v = m.area_v[g.ij(i, j)];
  // transports of momentum_advection.f90:13-19 at (ii, jj, k)
  auto utr = [&](int ii, int jj, int k) {
    return m.dzt[k - 1] * m.dyt[jj + 1] * ut[g.k3(ii, jj, k)] * m.maskU[g.k3(ii, jj, k)];
  };
  auto vtr = [&](int ii, int jj, int k) {
    return m.dzt[k - 1] * m.cosu[jj + 1] * m.dxt[ii + 1] * vt[g.k3(ii, jj, k)] * m.maskV[g.k3(ii, jj, k)];
  };
  auto wtr = [&](int ii, int jj, int k) {
    return m.area_t[g.ij(ii, jj)] * wt[g.k3(ii, jj, k)] * m.maskW[g.k3(ii, jj, k)];
  };
  double ftu_prev = 0.0, ftv_prev = 0.0;  // flux_top(k-1) of the u and v equations
  for (int k = 1; k <= nz; k++) {
    const size_t c = g.k3(i, j, k);
    const double mU = m.maskU[c], mV = m.maskV[c];
    // Coriolis (momentum.f90:13-16)
    double du_cor = mU *
                    (m.coriolis_t[g.ij(i, j)] * (vt[g.k3(i, j, k)] + vt[g.k3(i, j - 1, k)]) * dxt_i / dxu_i +
                     m.coriolis_t[g.ij(i + 1, j)] * (vt[g.k3(i + 1, j, k)] + vt[g.k3(i + 1, j - 1, k)]) * dxt_ip /
                         dxu_i) *
                    0.25;
    double dv_cor = -mV *
                    (m.coriolis_t[g.ij(i, j)] * (ut[g.k3(i - 1, j, k)] + ut[g.k3(i, j, k)]) * dyt_j * cost_j /
                         (dyu_j * cosu_j) +
                     m.coriolis_t[g.ij(i, j + 1)] * (ut[g.k3(i - 1, j + 1, k)] + ut[g.k3(i, j + 1, k)]) * dyt_jp *
                         cost_jp / (dyu_j * cosu_j)) *
                    0.25;
    if (m.coord_degree) {  // metric terms (momentum.f90:19-30)
      du_cor = du_cor + mU * 0.125 * m.tantr[j + 1] *
                            ((ut[g.k3(i, j, k)] + ut[g.k3(i - 1, j, k)]) * (vt[g.k3(i, j, k)] + vt[g.k3(i, j - 1, k)]) *
                                 dxt_i / dxu_i +
                             (ut[g.k3(i + 1, j, k)] + ut[g.k3(i, j, k)]) *
                                 (vt[g.k3(i + 1, j, k)] + vt[g.k3(i + 1, j - 1, k)]) * dxt_ip / dxu_i);
      const double s0 = ut[g.k3(i, j, k)] + ut[g.k3(i - 1, j, k)];
      const double s1 = ut[g.k3(i, j + 1, k)] + ut[g.k3(i - 1, j + 1, k)];
      dv_cor = dv_cor - mV * 0.125 *
                            (m.tantr[j + 1] * (s0 * s0) * dyt_j * cost_j / (dyu_j * cosu_j) +
                             m.tantr[j + 2] * (s1 * s1) * dyt_jp * cost_jp / (dyu_j * cosu_j));
    }
    double du_t = du_cor, dv_t = dv_cor;  // du(i,j,:,tau) = du_cor (:82-87)
    if (k == nz) {                        // wind stress (:89-93)
      du_t = du_t + mU * m.taux[g.ij(i, j)] / m.dzt[nz - 1];
      dv_t = dv_t + mV * m.tauy[g.ij(i, j)] / m.dzt[nz - 1];
    }
    // advection of u (momentum_advection.f90:22-45)
    {
      const double fe = 0.25 * (ut[g.k3(i, j, k)] + ut[g.k3(i + 1, j, k)]) * (utr(i + 1, j, k) + utr(i, j, k));
      const double fw = 0.25 * (ut[g.k3(i - 1, j, k)] + ut[g.k3(i, j, k)]) * (utr(i, j, k) + utr(i - 1, j, k));
      const double fn = 0.25 * (ut[g.k3(i, j, k)] + ut[g.k3(i, j + 1, k)]) * (vtr(i + 1, j, k) + vtr(i, j, k));
      const double fs =
          0.25 * (ut[g.k3(i, j - 1, k)] + ut[g.k3(i, j, k)]) * (vtr(i + 1, j - 1, k) + vtr(i, j - 1, k));
      double adv = -(mU * (fe - fw + fn - fs) / (area_u * m.dzt[k - 1]));
      const double ft =
          k < nz ? 0.25 * (ut[g.k3(i, j, k + 1)] + ut[g.k3(i, j, k)]) * (wtr(i, j, k) + wtr(i + 1, j, k)) : 0.0;
      if (k == 1)
        adv = adv - mU * ft / (area_u * m.dzt[k - 1]);
      else
        adv = adv - mU * (ft - ftu_prev) / (area_u * m.dzt[k - 1]);
      ftu_prev = ft;
      du_t = du_t + adv;
    }
    // advection of v (:46-69)
    {
      const double fe = 0.25 * (vt[g.k3(i, j, k)] + vt[g.k3(i + 1, j, k)]) * (utr(i, j + 1, k) + utr(i, j, k));
      const double fw =
          0.25 * (vt[g.k3(i - 1, j, k)] + vt[g.k3(i, j, k)]) * (utr(i - 1, j + 1, k) + utr(i - 1, j, k));
      const double fn = 0.25 * (vt[g.k3(i, j, k)] + vt[g.k3(i, j + 1, k)]) * (vtr(i, j + 1, k) + vtr(i, j, k));
      const double fs = 0.25 * (vt[g.k3(i, j - 1, k)] + vt[g.k3(i, j, k)]) * (vtr(i, j, k) + vtr(i, j - 1, k));
      double adv = -(mV * (fe - fw + fn - fs) / (area_v * m.dzt[k - 1]));
      const double ft =
          k < nz ? 0.25 * (vt[g.k3(i, j, k + 1)] + vt[g.k3(i, j, k)]) * (wtr(i, j, k) + wtr(i, j + 1, k)) : 0.0;
      if (k == 1)
        adv = adv - mV * ft / (area_v * m.dzt[k - 1]);
      else
        adv = adv - mV * (ft - ftv_prev) / (area_v * m.dzt[k - 1]);
      ftv_prev = ft;
      dv_t = dv_t + adv;
    }
    m.du[g.k4(i, j, k, tau)] = du_t;
    m.dv[g.k4(i, j, k, tau)] = dv_t;
  }
}

// ---- implicit vertical friction (vertical_friction.f90:109-226) ------------------
// For the u (uv = 0) or v (uv = 1) point (i, j): the tridiagonal system of its
// column with the viscosity kappaM averaged onto the point, solved as
// solve_tridiag does (numerics.f90:548-581) into u(:,:,:,taup1) (the
// reference's scratch), then du_mix = (u(taup1) - u(tau)) / dt_mom.
constexpr int kMaxNz = 128;

__global__ void k_mom_implicit(MomDev m, int uv) {
  const MG& g = m.g;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nx * g.ny) return;
  const int i = 1 + t % g.nx, j = 1 + t / g.nx;
  const int nz = g.nz;
  const int i1 = uv == 0 ? i + 1 : i, j1 = uv == 0 ? j : j + 1;  // the neighbour sharing the point
  const double* mask = uv == 0 ? m.maskU : m.maskV;
  double* q = uv == 0 ? m.u : m.v;
  double* q_mix = uv == 0 ? m.du_mix : m.dv_mix;
  const double* qt = q + (size_t)(m.tau - 1) * g.n2 * nz;
  double* qn = q + (size_t)(m.taup1 - 1) * g.n2 * nz;
  if (!m.implicit_vert) {
    for (int k = 1; k <= nz; k++) q_mix[g.k3(i, j, k)] = 0.0;  // momentum.f90:115-117
    return;
  }
  const int ks = max(m.kbot[g.ij(i, j)], m.kbot[g.ij(i1, j1)]);
  if (ks > 0 && ks < nz) {
    double delta[kMaxNz], cp[kMaxNz], dp[kMaxNz];
    for (int k = ks; k <= nz - 1; k++) {
      const double fxa = 0.5 * (m.kappaM[g.k3(i, j, k)] + m.kappaM[g.k3(i1, j1, k)]);
      delta[k - 1] = m.dt_mom / m.dzw[k - 1] * fxa * mask[g.k3(i, j, k + 1)] * mask[g.k3(i, j, k)];
    }
    delta[nz - 1] = 0.0;
    // a, b, c of :128-141
    auto a = [&](int k) { return k == ks ? 0.0 : -delta[k - 2] / m.dzt[k - 1]; };
    auto b = [&](int k) {
      if (k == nz) return 1 + delta[nz - 2] / m.dzt[nz - 1];
      if (k == ks) return 1 + delta[k - 1] / m.dzt[k - 1];
      return 1 + delta[k - 1] / m.dzt[k - 1] + delta[k - 2] / m.dzt[k - 1];
    };
    auto cc = [&](int k) { return k == nz ? 0.0 : -delta[k - 1] / m.dzt[k - 1]; };
    cp[ks - 1] = cc(ks) / b(ks);
    dp[ks - 1] = qt[g.k3(i, j, ks)] / b(ks);
    for (int k = ks + 1; k <= nz; k++) {
      const double mm = b(k) - cp[k - 2] * a(k);
      const double fxa = 1.0 / mm;
      cp[k - 1] = cc(k) * fxa;
      dp[k - 1] = (qt[g.k3(i, j, k)] - dp[k - 2] * a(k)) * fxa;
    }
    double x = dp[nz - 1];
    qn[g.k3(i, j, nz)] = x;
    for (int k = nz - 1; k >= ks; k--) {
      x = dp[k - 1] - cp[k - 1] * x;
      qn[g.k3(i, j, k)] = x;
    }
  } else if (ks == nz) {
    // one wet cell: the reference's b(nz) reads delta(nz-1) left over from an
    // earlier column (vertical_friction.f90:135); without coupling the cell
    // keeps its velocity here
    qn[g.k3(i, j, nz)] = qt[g.k3(i, j, nz)];
  }
  for (int k = 1; k <= nz; k++) q_mix[g.k3(i, j, k)] = (qn[g.k3(i, j, k)] - qt[g.k3(i, j, k)]) / m.dt_mom;
}

// ---- harmonic lateral friction and linear bottom friction -> du_mix, dv_mix ------
// harmonic_friction.f90:11-39 (u) and :69-94 (v); bottom_friction.f90:110-135.
__global__ void k_mom_lateral(MomDev m) {
  const MG& g = m.g;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nx * g.ny) return;
  const int i = 1 + t % g.nx, j = 1 + t / g.nx;
  const int nz = g.nz, tau = m.tau;
  const double* ut = m.u + (size_t)(tau - 1) * g.n2 * nz;
  const double* vt = m.v + (size_t)(tau - 1) * g.n2 * nz;
  const double A = m.A_h;
  const int pw = m.cos_power;
  const bool cs = m.cos_scaling;
  // the fluxes of harmonic_friction.f90 across the faces of point (ii, jj)
  auto fe_u = [&](int ii, int jj, int k) {  // flux_east of u
    const double d = (ut[g.k3(ii + 1, jj, k)] - ut[g.k3(ii, jj, k)]);
    const double den = m.cost[jj + 1] * m.dxt[ii + 2];
    const double r = cs ? ipow(m.cost[jj + 1], pw) * A * d / den : A * d / den;
    return r * m.maskU[g.k3(ii + 1, jj, k)] * m.maskU[g.k3(ii, jj, k)];
  };
  auto fn_u = [&](int ii, int jj, int k) {  // flux_north of u
    const double d = (ut[g.k3(ii, jj + 1, k)] - ut[g.k3(ii, jj, k)]);
    const double r = cs ? ipow(m.cosu[jj + 1], pw) * A * d / m.dyu[jj + 1] : A * d / m.dyu[jj + 1];
    return r * m.maskU[g.k3(ii, jj + 1, k)] * m.maskU[g.k3(ii, jj, k)] * m.cosu[jj + 1];
  };
  auto fe_v = [&](int ii, int jj, int k) {
    const double d = (vt[g.k3(ii + 1, jj, k)] - vt[g.k3(ii, jj, k)]);
    const double den = m.cosu[jj + 1] * m.dxu[ii + 1];
    const double r = cs ? ipow(m.cosu[jj + 1], pw) * A * d / den : A * d / den;
    return r * m.maskV[g.k3(ii + 1, jj, k)] * m.maskV[g.k3(ii, jj, k)];
  };
  auto fn_v = [&](int ii, int jj, int k) {
    const double d = (vt[g.k3(ii, jj + 1, k)] - vt[g.k3(ii, jj, k)]);
    const double r = cs ? ipow(m.cost[jj + 2], pw) * A * d / m.dyt[jj + 2] : A * d / m.dyt[jj + 2];
    return r * m.cost[jj + 2] * m.maskV[g.k3(ii, jj, k)] * m.maskV[g.k3(ii, jj + 1, k)];
  };
  const int kbu = max(m.kbot[g.ij(i, j)], m.kbot[g.ij(i + 1, j)]);
  const int kbv = max(m.kbot[g.ij(i, j + 1)], m.kbot[g.ij(i, j)]);
  for (int k = 1; k <= nz; k++) {
    const size_t c = g.k3(i, j, k);
    double dum = m.du_mix[c], dvm = m.dv_mix[c];
    if (m.hor_friction) {
      dum = dum + m.maskU[c] * ((fe_u(i, j, k) - fe_u(i - 1, j, k)) / (m.cost[j + 1] * m.dxu[i + 1]) +
                                (fn_u(i, j, k) - fn_u(i, j - 1, k)) / (m.cost[j + 1] * m.dyt[j + 1]));
      dvm = dvm + m.maskV[c] * ((fe_v(i, j, k) - fe_v(i - 1, j, k)) / (m.cosu[j + 1] * m.dxt[i + 1]) +
                                (fn_v(i, j, k) - fn_v(i, j - 1, k)) / (m.dyu[j + 1] * m.cosu[j + 1]));
    }
    if (m.bottom_friction) {
      if (k == kbu) dum = dum - m.maskU[c] * m.r_bot * ut[c];
      if (k == kbv) dvm = dvm - m.maskV[c] * m.r_bot * vt[c];
    }
    m.du_mix[c] = dum;
    m.dv_mix[c] = dvm;
  }
}

// ---- the cyclic halo copies of u and v at time level lev (parallel_none.f90:
// setcyclic_xyz; the reference's time loop does them at main.f90:114-117) -----------
__global__ void k_setcyclic_uv(MomDev m, int lev, int cyclic_x, int cyclic_y) {
  const MG& g = m.g;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nrow = g.ny + 4;  // j = -1 .. ny+2
  if (t >= 2 * nrow * g.nz) return;
  const int f = t / (nrow * g.nz), r = t % (nrow * g.nz);
  const int j = r % nrow - 1, k = 1 + r / nrow;
  double* a = (f == 0 ? m.u : m.v) + (size_t)(lev - 1) * g.n2 * g.nz;
  if (cyclic_x)
    for (int i = 1; i <= 2; i++) {
      a[g.k3(g.nx + i, j, k)] = a[g.k3(i, j, k)];
      a[g.k3(1 - i, j, k)] = a[g.k3(g.nx - i + 1, j, k)];
    }
  (void)cyclic_y;
}

// rows of a cyclic-y domain, after every column has its x copies
__global__ void k_setcyclic_uv_y(MomDev m, int lev) {
  const MG& g = m.g;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = g.nx + 4;  // i = -1 .. nx+2
  if (t >= 2 * ncol * g.nz) return;
  const int f = t / (ncol * g.nz), r = t % (ncol * g.nz);
  const int i = r % ncol - 1, k = 1 + r / ncol;
  double* a = (f == 0 ? m.u : m.v) + (size_t)(lev - 1) * g.n2 * g.nz;
  for (int j = 1; j <= 2; j++) {
    a[g.k3(i, g.ny + j, k)] = a[g.k3(i, j, k)];
    a[g.k3(i, 1 - j, k)] = a[g.k3(i, g.ny - j + 1, k)];
  }
}

// ---- vertical_velocity (vertical_velocity.f90:4-25) at time level lev --------------
__global__ void k_vertical_velocity(MomDev m, int lev) {
  const MG& g = m.g;
  const int W = g.nx + 3, H = g.ny + 3;  // i = 0 .. nx+2, j = 0 .. ny+2
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= W * H) return;
  const int i = t % W, j = t / W;
  const double* ul = m.u + (size_t)(lev - 1) * g.n2 * g.nz;
  const double* vl = m.v + (size_t)(lev - 1) * g.n2 * g.nz;
  double* wl = m.w + (size_t)(lev - 1) * g.n2 * g.nz;
  const double ct = m.cost[j + 1], dx = m.dxt[i + 1], dy = m.dyt[j + 1], cu = m.cosu[j + 1], cum = m.cosu[j];
  double prev = 0.0;
  for (int k = 1; k <= g.nz; k++) {
    const double div = (ul[g.k3(i, j, k)] - ul[g.k3(i - 1, j, k)]) / (ct * dx) +
                       (cu * vl[g.k3(i, j, k)] - cum * vl[g.k3(i, j - 1, k)]) / (ct * dy);
    const double wk = k == 1 ? -m.maskW[g.k3(i, j, k)] * m.dzt[k - 1] * div
                             : prev - m.maskW[g.k3(i, j, k)] * m.dzt[k - 1] * div;
    wl[g.k3(i, j, k)] = wk;
    prev = wk;
  }
}

MomDev to_dev(const pyomgpu_momentum* p, int nx, int ny, const double* const* g1) {
  MomDev m{};
  m.g = MG{nx, ny, p->nz, (size_t)(nx + 4) * (ny + 4)};
  m.tau = p->tau;
  m.taup1 = p->taup1;
  m.coord_degree = p->coord_degree;
  m.hor_friction = p->enable_hor_friction;
  m.cos_scaling = p->enable_hor_friction_cos_scaling;
  m.cos_power = p->hor_friction_cospower;
  m.bottom_friction = p->enable_bottom_friction;
  m.implicit_vert = p->enable_implicit_vert_friction;
  m.dt_mom = p->dt_mom;
  m.A_h = p->A_h;
  m.r_bot = p->r_bot;
  m.dxt = g1[0];
  m.dxu = g1[1];
  m.dyt = g1[2];
  m.dyu = g1[3];
  m.cost = g1[4];
  m.cosu = g1[5];
  m.tantr = p->tantr;
  m.dzt = p->dzt;
  m.dzw = p->dzw;
  m.maskU = p->maskU;
  m.maskV = p->maskV;
  m.maskW = p->maskW;
  m.kappaM = p->kappaM;
  m.kbot = p->kbot;
  m.coriolis_t = p->coriolis_t;
  m.area_t = p->area_t;
  m.area_u = p->area_u;
  m.area_v = p->area_v;
  m.taux = p->surface_taux;
  m.tauy = p->surface_tauy;
  m.u = p->u;
  m.v = p->v;
  m.w = p->w;
  m.du = p->du;
  m.dv = p->dv;
  m.du_mix = p->du_mix;
  m.dv_mix = p->dv_mix;
  return m;
}

bool valid(const pyomgpu_momentum* p) {
  if (!p || p->nz < 2 || p->nz > kMaxNz || p->hor_friction_cospower < 0 || p->hor_friction_cospower > 8) return false;
  for (int t : {p->tau, p->taup1})
    if (t < 1 || t > 3) return false;
  if (p->tau == p->taup1 || p->dt_mom == 0.0) return false;
  const void* need[] = {p->dzt,    p->dzw,      p->tantr,  p->maskU,  p->maskV,  p->maskW,
                        p->kappaM, p->kbot,     p->coriolis_t, p->area_t, p->area_u, p->area_v,
                        p->surface_taux, p->surface_tauy, p->u, p->v, p->w, p->du, p->dv, p->du_mix, p->dv_mix};
  for (const void* q : need)
    if (!q) return false;
  return true;
}

}  // namespace
}  // namespace pyomgpu

using namespace pyomgpu;

extern "C" int32_t pyomgpu_momentum_tendencies(pyomgpu_ctx* c, const pyomgpu_momentum* p, pyomgpu_stream stream) {
  if (!c || !valid(p))
    return mfail(PYOMGPU_EINVAL, "momentum: bad arguments (nz in 2..128, distinct time levels, dt_mom != 0, "
                                 "every array given)");
  int nx = 0, ny = 0;
  const double* g1[6];
  if (int rc = ctx_grid1d(c, &nx, &ny, g1, nullptr, nullptr)) return rc;
  const MomDev m = to_dev(p, nx, ny, g1);
  cudaStream_t st = (cudaStream_t)stream;
  const int n = nx * ny, tb = 128, nb = (n + tb - 1) / tb;
  k_mom_cor_adv<<<nb, tb, 0, st>>>(m);
  k_mom_implicit<<<nb, tb, 0, st>>>(m, 0);
  k_mom_implicit<<<nb, tb, 0, st>>>(m, 1);
  k_mom_lateral<<<nb, tb, 0, st>>>(m);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mfail(PYOMGPU_ECUDA, "momentum kernels: %s", cudaGetErrorString(e));
  return PYOMGPU_OK;
}

extern "C" int32_t pyomgpu_vertical_velocity(pyomgpu_ctx* c, const pyomgpu_momentum* p, int32_t level,
                                            pyomgpu_stream stream) {
  if (!c || !p || !p->u || !p->v || !p->w || !p->maskW || !p->dzt || level < 1 || level > 3 || p->nz < 1)
    return mfail(PYOMGPU_EINVAL, "vertical_velocity: bad arguments");
  int nx = 0, ny = 0, cx = 0, cy = 0;
  const double* g1[6];
  if (int rc = ctx_grid1d(c, &nx, &ny, g1, &cx, &cy)) return rc;
  MomDev m{};
  m.g = MG{nx, ny, p->nz, (size_t)(nx + 4) * (ny + 4)};
  m.dxt = g1[0];
  m.dyt = g1[2];
  m.cost = g1[4];
  m.cosu = g1[5];
  m.dzt = p->dzt;
  m.maskW = p->maskW;
  m.u = p->u;
  m.v = p->v;
  m.w = p->w;
  const int tb = 128;
  cudaStream_t st = (cudaStream_t)stream;
  if (cx) {
    const int nr = 2 * (ny + 4) * p->nz;
    k_setcyclic_uv<<<(nr + tb - 1) / tb, tb, 0, st>>>(m, level, cx, cy);
  }
  if (cy) {
    const int nc = 2 * (nx + 4) * p->nz;
    k_setcyclic_uv_y<<<(nc + tb - 1) / tb, tb, 0, st>>>(m, level);
  }
  const int n = (nx + 3) * (ny + 3);
  k_vertical_velocity<<<(n + tb - 1) / tb, tb, 0, st>>>(m, level);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mfail(PYOMGPU_ECUDA, "vertical_velocity: %s", cudaGetErrorString(e));
  return PYOMGPU_OK;
}
