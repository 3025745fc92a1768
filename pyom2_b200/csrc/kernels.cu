// Operator construction, layout conversion, island integrals and the
// column-wise pre/post work of one external-mode step.
#include <math.h>

#include <algorithm>

#include "kernels.cuh"

namespace pyomgpu {

namespace {

inline unsigned nblk(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// Fortran halo index range of a padded field: i in [-1, nx+2], j in [-1, ny+2].
__device__ __forceinline__ bool decode_full(const Geo& g, size_t t, int& i, int& j) {
  const int X = g.nx + 2 * kOnx, Y = g.ny + 2 * kOnx;
  if (t >= (size_t)X * Y) return false;
  i = (int)(t % X) - 1;
  j = (int)(t / X) - 1;
  return true;
}

// Source position of (i,j) after setcyclic_xy (parallel_none.f90:188-211).
__device__ __forceinline__ void cyclic_source(const Geo& g, int i, int j, int& si, int& sj) {
  si = i;
  sj = j;
  if (g.cyclic_x) {
    if (i < 1) si = i + g.nx;
    if (i > g.nx) si = i - g.nx;
  }
  if (g.cyclic_y) {
    if (j < 1) sj = j + g.ny;
    if (j > g.ny) sj = j - g.ny;
  }
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
__global__ void k_build_sf(GridDev gd, Geo g, double* FX, double* FY, double* ax, double* bx, double* by) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  const int nx = g.nx;
  double fx = 0.0, fy = 0.0;
  // solve_streamfct.f90:137-140 : E/W couplings hvr(i,j)/dxt(i), i = 1..nx+1
  if (i >= 1 && i <= g.nx + 1 && j >= 1 && j <= g.ny) fx = gd.hvr[fidx(nx, i, j)] / gd.dxt[i + 1];
  // :142-145 : N/S couplings hur(i,j) cost(j)/dyt(j), j = 1..ny+1
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny + 1) fy = gd.hur[fidx(nx, i, j)] * gd.cost[j + 1] / gd.dyt[j + 1];
  FX[g.at(i, j)] = fx;
  FY[g.at(i, j)] = fy;
  if (j == -1) ax[i + 1] = 1.0 / gd.dxu[i + 1];
  if (i == -1) {
    const double cu = gd.cosu[j + 1];
    bx[j + 1] = 1.0 / (cu * cu);
    by[j + 1] = 1.0 / (gd.dyu[j + 1] * cu);
  }
}

__global__ void k_build_sp(GridDev gd, Geo g, double* FX, double* FY, double* W, double* ax, double* bx,
                           double* by) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  const int nx = g.nx;
  const double* m = gd.maskT_top;
  double fx = 0.0, fy = 0.0;
  // solve_pressure.f90:109-114 : mp*hu(i,j)/dxu(i) between T(i) and T(i+1); stored at face i+1
  if (i >= 1 && i <= g.nx + 1 && j >= 1 && j <= g.ny)
    fx = m[fidx(nx, i - 1, j)] * m[fidx(nx, i, j)] * gd.hu[fidx(nx, i - 1, j)] / gd.dxu[i];
  // :116-121 : mp*hv(i,j)*cosu(j)/dyu(j) between T(j) and T(j+1); stored at face j+1
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny + 1)
    fy = m[fidx(nx, i, j - 1)] * m[fidx(nx, i, j)] * gd.hv[fidx(nx, i, j - 1)] * gd.cosu[j] / gd.dyu[j];
  FX[g.at(i, j)] = fx;
  FY[g.at(i, j)] = fy;
  W[g.at(i, j)] = m[fidx(nx, i, j)];
  if (j == -1) ax[i + 1] = 1.0 / gd.dxt[i + 1];
  if (i == -1) {
    const double ct = gd.cost[j + 1];
    bx[j + 1] = 1.0 / (ct * ct);
    by[j + 1] = 1.0 / (gd.dyt[j + 1] * ct);
  }
}

// make_inv_sfc (solve_streamfct.f90:394-411): Z = 1/cf(i,j,2,2) or 0.
__global__ void k_inv_diag(Geo g, OpDev<double> op, double* Z) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  double z = 0.0;
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) {
    const double sx = op.ax[i + 1] * op.bx[j + 1];
    const double sy = op.by[j + 1];
    const double c = -(sx * (op.FX[g.at(i + 1, j)] + op.FX[g.at(i, j)]) + sy * (op.FY[g.at(i, j + 1)] + op.FY[g.at(i, j)]));
    z = (c != 0.0) ? 1.0 / c : 0.0;
  }
  Z[g.at(i, j)] = z;
}

// make_inv_sfc :415-421 -- zero on island perimeter points (interior ones; the
// halo of the reference's Z is zero anyway and ours holds cyclic copies).
__global__ void k_zero_points(Geo g, double* Z, const int* pi, const int* pj, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = pi[t], j = pj[t];
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) Z[g.at(i, j)] = 0.0;
}

// Fill halo cells of a padded field from the interior (setcyclic_xy).
__global__ void k_fill_cyclic_padded(Geo g, double* a) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) return;
  int si, sj;
  cyclic_source(g, i, j, si, sj);
  if (si == i && sj == j) return;
  if (si < 1 || si > g.nx || sj < 1 || sj > g.ny) return;  // halo row of a non-cyclic direction
  a[g.at(i, j)] = a[g.at(si, sj)];
}

// ---------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------
__global__ void k_pack(Geo g, const double* __restrict__ user, double* __restrict__ pad, int setcyc) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  int si = i, sj = j;
  if (setcyc) cyclic_source(g, i, j, si, sj);
  pad[g.at(i, j)] = user[fidx(g.nx, si, sj)];
}

__global__ void k_unpack(Geo g, const double* __restrict__ pad, double* __restrict__ user, int setcyc,
                         int interior_only, int zero_halo) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  const bool inner = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
  if (interior_only && !inner) return;
  if (zero_halo && !inner) {
    user[fidx(g.nx, i, j)] = 0.0;
    return;
  }
  int si = i, sj = j;
  if (setcyc) cyclic_source(g, i, j, si, sj);
  user[fidx(g.nx, i, j)] = pad[g.at(si, sj)];
}

// setcyclic_xy on a Fortran-layout array; x pass then y pass as the reference.
__global__ void k_setcyclic_user_x(int nx, int ny, double* a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x - 1;
  if (j > ny + 2) return;
  for (int i = 1; i <= kOnx; i++) {
    a[fidx(nx, nx + i, j)] = a[fidx(nx, i, j)];
    a[fidx(nx, 1 - i, j)] = a[fidx(nx, nx - i + 1, j)];
  }
}
__global__ void k_setcyclic_user_y(int nx, int ny, double* a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1;
  if (i > nx + 2) return;
  for (int j = 1; j <= kOnx; j++) {
    a[fidx(nx, i, ny + j)] = a[fidx(nx, i, j)];
    a[fidx(nx, i, 1 - j)] = a[fidx(nx, i, ny - j + 1)];
  }
}

__global__ void k_apply_user(Geo g, OpDev<double> op, const double* __restrict__ pad, double* __restrict__ res) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  double r = 0.0;
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny) r = apply_point(op, g, pad, i, j);
  res[fidx(g.nx, i, j)] = r;
}

// ---------------------------------------------------------------------------
// island integrals (streamfct_init.f90:311-377)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double seg_contrib(int nx, const LineGeo& lg, int d, int i, int j, double u_ij,
                                              double u_ijp, double v_ij, double v_ipj) {
  switch (d) {
    case 0:  // to east  (:339)
      return v_ij * lg.dyu[j + 1] + u_ijp * lg.dxu[i + 1] * lg.cost[j + 2];
    case 1:  // to west  (:348)
      return -v_ipj * lg.dyu[j + 1] - u_ij * lg.dxu[i + 1] * lg.cost[j + 1];
    case 2:  // to north (:357)
      return v_ij * lg.dyu[j + 1] - u_ij * lg.dxu[i + 1] * lg.cost[j + 1];
    default:  // to south (:366)
      return u_ijp * lg.dxu[i + 1] * lg.cost[j + 2] - v_ipj * lg.dyu[j + 1];
  }
}

constexpr int kLineThreads = 256;

__global__ void __launch_bounds__(kLineThreads) k_line_uv(int nx, IslandDev isl, LineGeo lg, const double* u,
                                                          const double* v, int k0, double* out) {
  const int k = k0 + blockIdx.x;
  double acc = 0.0;
  for (int s = isl.seg_off[k] + threadIdx.x; s < isl.seg_off[k + 1]; s += kLineThreads) {
    const int i = isl.seg_i[s], j = isl.seg_j[s], d = isl.seg_d[s];
    acc += seg_contrib(nx, lg, d, i, j, u[fidx(nx, i, j)], u[fidx(nx, i, j + 1)], v[fidx(nx, i, j)],
                       v[fidx(nx, i + 1, j)]);
  }
  double vv[1] = {acc}, o[1];
  block_reduce<1, -1, kLineThreads>(vv, o);
  if (threadIdx.x == 0) out[blockIdx.x] = o[0];
}

// velocity of a streamfunction: streamfct_init.f90:297-298, solve_streamfct.f90:71-72
__device__ __forceinline__ double psi_u(int nx, const LineGeo& lg, const double* p, int i, int j) {
  return -lg.maskU_top[fidx(nx, i, j)] * (p[fidx(nx, i, j)] - p[fidx(nx, i, j - 1)]) / lg.dyt[j + 1] *
         lg.hur[fidx(nx, i, j)];
}
__device__ __forceinline__ double psi_v(int nx, const LineGeo& lg, const double* p, int i, int j) {
  return lg.maskV_top[fidx(nx, i, j)] * (p[fidx(nx, i, j)] - p[fidx(nx, i - 1, j)]) / (lg.cosu[j + 1] * lg.dxt[i + 1]) *
         lg.hvr[fidx(nx, i, j)];
}

__global__ void __launch_bounds__(kLineThreads) k_line_psi(int nx, IslandDev isl, LineGeo lg, const double* psi,
                                                           size_t stride, int k0, int nk, double* out) {
  const int k = k0 + blockIdx.x;
  const int f = blockIdx.y;
  const double* p = psi + (size_t)f * stride;
  double acc = 0.0;
  for (int s = isl.seg_off[k] + threadIdx.x; s < isl.seg_off[k + 1]; s += kLineThreads) {
    const int i = isl.seg_i[s], j = isl.seg_j[s], d = isl.seg_d[s];
    acc += seg_contrib(nx, lg, d, i, j, psi_u(nx, lg, p, i, j), psi_u(nx, lg, p, i, j + 1), psi_v(nx, lg, p, i, j),
                       psi_v(nx, lg, p, i + 1, j));
  }
  double vv[1] = {acc}, o[1];
  block_reduce<1, -1, kLineThreads>(vv, o);
  if (threadIdx.x == 0) out[(size_t)f * nk + blockIdx.x] = o[0];
}

// DGETRS with the host factors (solve_streamfct.f90:77-87).  One thread; the
// island system is small (nisle - 1 unknowns).
__global__ void k_island_solve(int nisle, const double* lu, const int* ipiv, const double* lf, const double* lp,
                               double* dpsin, int tau) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int m = nisle - 1;
  extern __shared__ double b[];
  for (int k = 0; k < m; k++) b[k] = lf[k] - lp[k];
  for (int k = 0; k < m; k++) {
    const int p = ipiv[k] - 1;
    if (p != k) {
      const double t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
  }
  for (int c = 0; c < m; c++)
    for (int r = c + 1; r < m; r++) b[r] = b[r] - lu[(size_t)r + (size_t)c * m] * b[c];
  for (int c = m - 1; c >= 0; c--) {
    b[c] = b[c] / lu[(size_t)c + (size_t)c * m];
    for (int r = 0; r < c; r++) b[r] = b[r] - lu[(size_t)r + (size_t)c * m] * b[c];
  }
  for (int k = 0; k < m; k++) dpsin[(size_t)(k + 1) + (size_t)(tau - 1) * nisle] = b[k];
}

// ---------------------------------------------------------------------------
// step pre/post (solve_streamfct.f90:24-53,91-118; solve_pressure.f90:19-80)
// ---------------------------------------------------------------------------
__device__ __forceinline__ size_t q3(const StepDev& s, size_t q2, int k) {
  return q2 + (size_t)(k - 1) * (size_t)(s.nx + 4) * (s.ny + 4);
}
__device__ __forceinline__ size_t q4(const StepDev& s, size_t q2, int k, int t) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  return q2 + (size_t)(k - 1) * n2 + (size_t)(t - 1) * n2 * s.nz;
}

__global__ void k_hydrostatic(StepDev s) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const double fxa = s.grav / s.rho_0;
  const int nz = s.nz;
  double ph = 0.5 * s.rho[q4(s, q, nz, s.tau)] * fxa * s.dzw[nz - 1] * s.maskT[q3(s, q, nz)];
  s.p_hydro[q3(s, q, nz)] = ph;
  double rk1 = s.rho[q4(s, q, nz, s.tau)];
  for (int k = nz - 1; k >= 1; k--) {
    const double rk = s.rho[q4(s, q, k, s.tau)];
    ph = s.maskT[q3(s, q, k)] * (ph + 0.5 * (rk1 + rk) * fxa * s.dzw[k - 1]);
    s.p_hydro[q3(s, q, k)] = ph;
    rk1 = rk;
  }
}

__global__ void k_sf_columns(StepDev s, double* fpx, double* fpy) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int i = (int)(q % (s.nx + 4)) - 1, j = (int)(q / (s.nx + 4)) - 1;
  const bool inner = i >= 1 && i <= s.nx && j >= 1 && j <= s.ny;
  const size_t qe = fidx(s.nx, i + 1, j), qn = fidx(s.nx, i, j + 1);
  double ax = 0.0, ay = 0.0;
  for (int k = 1; k <= s.nz; k++) {
    const size_t d = q4(s, q, k, s.tau);
    double du = s.du[d], dv = s.dv[d];
    if (inner) {  // solve_streamfct.f90:32-37
      du = du - (s.p_hydro[q3(s, qe, k)] - s.p_hydro[q3(s, q, k)]) / (s.dxu[i + 1] * s.cost[j + 1]) * s.maskU[q3(s, q, k)];
      dv = dv - (s.p_hydro[q3(s, qn, k)] - s.p_hydro[q3(s, q, k)]) / s.dyu[j + 1] * s.maskV[q3(s, q, k)];
      s.du[d] = du;
      s.dv[d] = dv;
    }
    // :40-43
    ax = ax + (du + s.du_mix[q3(s, q, k)]) * s.maskU[q3(s, q, k)] * s.dzt[k - 1];
    ay = ay + (dv + s.dv_mix[q3(s, q, k)]) * s.maskV[q3(s, q, k)] * s.dzt[k - 1];
  }
  fpx[q] = ax * s.hur[q];  // :44
  fpy[q] = ay * s.hvr[q];
}

__global__ void k_sf_forc(StepDev s, const double* fpx, const double* fpy, double* forc) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int i = (int)(q % (s.nx + 4)) - 1, j = (int)(q / (s.nx + 4)) - 1;
  double f = 0.0;
  if (i >= 1 && i <= s.nx && j >= 1 && j <= s.ny)  // :49-53
    f = (fpy[fidx(s.nx, i + 1, j)] - fpy[q]) / (s.cosu[j + 1] * s.dxu[i + 1]) -
        (s.cost[j + 2] * fpx[fidx(s.nx, i, j + 1)] - s.cost[j + 1] * fpx[q]) / (s.cosu[j + 1] * s.dyu[j + 1]);
  forc[q] = f;
}

__global__ void k_first_guess(size_t n2, double* a1, const double* a0, const double* am) {
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q < n2) a1[q] = 2 * a0[q] - am[q];
}

__global__ void k_sf_psi(StepDev s, const double* psin, int nisle, const double* dpsin) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const double AB = s.AB_eps, dt = s.dt_mom;
  const double* ps0 = s.psi + (size_t)(s.tau - 1) * n2;
  double* ps1 = s.psi + (size_t)(s.taup1 - 1) * n2;
  const double* dp1 = s.dpsi + (size_t)(s.taup1 - 1) * n2;
  const double* dp0 = s.dpsi + (size_t)(s.tau - 1) * n2;
  double p = ps0[q] + dt * ((1.5 + AB) * dp1[q] - (0.5 + AB) * dp0[q]);  // :91
  for (int isle = 2; isle <= nisle; isle++) {                                // :92-94
    const double c = dt * ((1.5 + AB) * dpsin[(size_t)(isle - 1) + (size_t)(s.tau - 1) * nisle] -
                           (0.5 + AB) * dpsin[(size_t)(isle - 1) + (size_t)(s.taum1 - 1) * nisle]);
    p = p + c * psin[q + (size_t)(isle - 1) * n2];
  }
  ps1[q] = p;
}

__global__ void k_sf_velocity(StepDev s) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int i = (int)(q % (s.nx + 4)) - 1, j = (int)(q / (s.nx + 4)) - 1;
  const double AB = s.AB_eps, dt = s.dt_mom;
  double ax = 0.0, ay = 0.0;
  for (int k = 1; k <= s.nz; k++) {  // :95-96 and :102-106
    const size_t a1 = q4(s, q, k, s.taup1), a0 = q4(s, q, k, s.tau), am = q4(s, q, k, s.taum1), m = q3(s, q, k);
    const double un = s.u[a0] + dt * (s.du_mix[m] + (1.5 + AB) * s.du[a0] - (0.5 + AB) * s.du[am]) * s.maskU[m];
    const double vn = s.v[a0] + dt * (s.dv_mix[m] + (1.5 + AB) * s.dv[a0] - (0.5 + AB) * s.dv[am]) * s.maskV[m];
    s.u[a1] = un;
    s.v[a1] = vn;
    ax = ax + un * s.maskU[m] * s.dzt[k - 1];
    ay = ay + vn * s.maskV[m] * s.dzt[k - 1];
  }
  const bool inner = i >= 1 && i <= s.nx && j >= 1 && j <= s.ny;
  const double* ps1 = s.psi + (size_t)(s.taup1 - 1) * n2;
  double gu = 0.0, gv = 0.0;
  if (inner) {
    gu = ps1[q] - ps1[fidx(s.nx, i, j - 1)];
    gv = ps1[q] - ps1[fidx(s.nx, i - 1, j)];
  }
  for (int k = 1; k <= s.nz; k++) {  // :107-118
    const size_t a1 = q4(s, q, k, s.taup1), m = q3(s, q, k);
    double un = s.u[a1] - ax * s.maskU[m] * s.hur[q];
    double vn = s.v[a1] - ay * s.maskV[m] * s.hvr[q];
    if (inner) {
      un = un - s.maskU[m] * gu / s.dyt[j + 1] * s.hur[q];
      vn = vn + s.maskV[m] * gv / (s.cosu[j + 1] * s.dxt[i + 1]) * s.hvr[q];
    }
    s.u[a1] = un;
    s.v[a1] = vn;
  }
}

__global__ void k_sp_columns(StepDev s, double* fpx, double* fpy) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int i = (int)(q % (s.nx + 4)) - 1, j = (int)(q / (s.nx + 4)) - 1;
  const bool inner = i >= 1 && i <= s.nx && j >= 1 && j <= s.ny;
  const size_t qe = fidx(s.nx, i + 1, j), qn = fidx(s.nx, i, j + 1);
  const double AB = s.AB_eps, dt = s.dt_mom;
  double ax = 0.0, ay = 0.0;
  for (int k = 1; k <= s.nz; k++) {
    const size_t d = q4(s, q, k, s.tau), m = q3(s, q, k);
    double du = s.du[d], dv = s.dv[d];
    if (inner) {  // solve_pressure.f90:27-32
      du = du - (s.p_hydro[q3(s, qe, k)] - s.p_hydro[m]) / (s.dxu[i + 1] * s.cost[j + 1]) * s.maskU[m];
      dv = dv - (s.p_hydro[q3(s, qn, k)] - s.p_hydro[m]) / s.dyu[j + 1] * s.maskV[m];
      s.du[d] = du;
      s.dv[d] = dv;
    }
    const size_t a1 = q4(s, q, k, s.taup1), a0 = d, am = q4(s, q, k, s.taum1);
    const double un = s.u[a0] + dt * (s.du_mix[m] + (1.5 + AB) * du - (0.5 + AB) * s.du[am]) * s.maskU[m];  // :36
    const double vn = s.v[a0] + dt * (s.dv_mix[m] + (1.5 + AB) * dv - (0.5 + AB) * s.dv[am]) * s.maskV[m];  // :37
    s.u[a1] = un;
    s.v[a1] = vn;
    if (inner) {  // :40-48
      ax = ax + un * s.maskU[m] * s.dzt[k - 1] / dt;
      ay = ay + vn * s.maskV[m] * s.dzt[k - 1] / dt;
    }
  }
  fpx[q] = ax;
  fpy[q] = ay;
}

__global__ void k_sp_forc(StepDev s, int free_surface, const double* fpx, const double* fpy, double* forc) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int i = (int)(q % (s.nx + 4)) - 1, j = (int)(q / (s.nx + 4)) - 1;
  double f = 0.0;
  if (i >= 1 && i <= s.nx && j >= 1 && j <= s.ny) {  // :55-59
    f = (fpx[q] - fpx[fidx(s.nx, i - 1, j)]) / (s.cost[j + 1] * s.dxt[i + 1]) +
        (s.cosu[j + 1] * fpy[q] - s.cosu[j] * fpy[fidx(s.nx, i, j - 1)]) / (s.cost[j + 1] * s.dyt[j + 1]);
    if (free_surface) {  // :60-66
      const double* ps0 = s.psi + (size_t)(s.tau - 1) * n2;
      f = f - ps0[q] / (s.grav * (s.dt_mom * s.dt_mom)) * s.maskT[q3(s, q, s.nz)];
    }
  }
  forc[q] = f;
}

__global__ void k_sp_velocity(StepDev s) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= n2) return;
  const int i = (int)(q % (s.nx + 4)) - 1, j = (int)(q / (s.nx + 4)) - 1;
  if (!(i >= 1 && i <= s.nx && j >= 1 && j <= s.ny)) return;
  const double* ps1 = s.psi + (size_t)(s.taup1 - 1) * n2;
  const double dt = s.dt_mom;
  const double gx = ps1[fidx(s.nx, i + 1, j)] - ps1[q];
  const double gy = ps1[fidx(s.nx, i, j + 1)] - ps1[q];
  for (int k = 1; k <= s.nz; k++) {  // :75-80
    const size_t a1 = q4(s, q, k, s.taup1), m = q3(s, q, k);
    s.u[a1] = s.u[a1] - dt * gx / (s.dxu[i + 1] * s.cost[j + 1]) * s.maskU[m];
    s.v[a1] = s.v[a1] - dt * gy / s.dyu[j + 1] * s.maskV[m];
  }
}

// ||forc - A sol||^2 and ||forc||^2 over the unknowns (W != 0), per block.
__global__ void k_residual(Geo g, OpDev<double> op, const double* __restrict__ forc_user,
                           const double* __restrict__ sol, double* __restrict__ part) {
  double rr = 0.0, bb = 0.0;
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx) + 1, j = (int)(t / g.nx) + 1;
    if (op.W[g.at(i, j)] == 0.0) continue;
    const double f = forc_user[fidx(g.nx, i, j)];
    const double r = f - apply_point(op, g, sol, i, j);
    rr += r * r;
    bb += f * f;
  }
  double v[2] = {rr, bb}, o[2];
  block_reduce<2, -1, 256>(v, o);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = o[0];
    part[2 * blockIdx.x + 1] = o[1];
  }
}
__global__ void k_residual_final(const double* part, int nb, double* out) {
  double rr = 0.0, bb = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) {
    rr += part[2 * b];
    bb += part[2 * b + 1];
  }
  rr = warp_sum(rr);
  bb = warp_sum(bb);
  if (threadIdx.x == 0) {
    out[0] = rr;
    out[1] = bb;
  }
}

// ---------------------------------------------------------------------------
// mixed precision: FP32 copies, scaled FP32 residual, FP64 correction
// ---------------------------------------------------------------------------
__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    b[t] = (float)a[t];
}

// b32 = s (forc - A x) at the unknowns (W != 0), 0 elsewhere; forc in Fortran layout
__global__ void k_residual_f32(Geo g, OpDev<double> op, const double* __restrict__ forc_user,
                               const double* __restrict__ x, double s, float* __restrict__ b32) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int i, j;
  if (!decode_full(g, t, i, j)) return;
  float v = 0.f;
  if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && op.W[g.at(i, j)] != 0.0)
    v = (float)(s * (forc_user[fidx(g.nx, i, j)] - apply_point(op, g, x, i, j)));
  b32[g.at(i, j)] = v;
}

// x += c e over the interior
__global__ void k_add_correction(Geo g, double* __restrict__ x, const float* __restrict__ e, double c) {
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx) + 1, j = (int)(t / g.nx) + 1;
    const size_t o = g.at(i, j);
    x[o] = x[o] + c * (double)e[o];
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static size_t full_count(const Geo& g) { return (size_t)(g.nx + 2 * kOnx) * (g.ny + 2 * kOnx); }

void launch_build_op_streamfunction(const GridDev& gd, const Geo& g, OpBuf& op, cudaStream_t st) {
  const size_t n = full_count(g);
  k_build_sf<<<nblk(n, 256), 256, 0, st>>>(gd, g, op.FX, op.FY, op.ax, op.bx, op.by);
  op.dcoef = 0.0;
}

void launch_build_op_surf_press(const GridDev& gd, const Geo& g, OpBuf& op, cudaStream_t st) {
  const size_t n = full_count(g);
  k_build_sp<<<nblk(n, 256), 256, 0, st>>>(gd, g, op.FX, op.FY, op.W, op.ax, op.bx, op.by);
}

void launch_build_inv_diag(const Geo& g, OpBuf& op, const int* bnd_i, const int* bnd_j, int nbnd, cudaStream_t st) {
  const size_t n = full_count(g);
  k_inv_diag<<<nblk(n, 256), 256, 0, st>>>(g, op.dev(), op.W);
  if (nbnd > 0) k_zero_points<<<nblk(nbnd, 256), 256, 0, st>>>(g, op.W, bnd_i, bnd_j, nbnd);
  if (g.cyclic_x || g.cyclic_y) k_fill_cyclic_padded<<<nblk(n, 256), 256, 0, st>>>(g, op.W);
}

void launch_pack(const Geo& g, const double* user, double* padded, bool setcyc, cudaStream_t st) {
  const size_t n = full_count(g);
  k_pack<<<nblk(n, 256), 256, 0, st>>>(g, user, padded, setcyc ? 1 : 0);
}

void launch_unpack(const Geo& g, const double* padded, double* user, bool setcyc, bool interior_only, bool zero_halo,
                   cudaStream_t st) {
  const size_t n = full_count(g);
  k_unpack<<<nblk(n, 256), 256, 0, st>>>(g, padded, user, setcyc ? 1 : 0, interior_only ? 1 : 0, zero_halo ? 1 : 0);
}

void launch_setcyclic_user(const Geo& g, double* user, cudaStream_t st) {
  if (g.cyclic_x) k_setcyclic_user_x<<<nblk(g.ny + 4, 128), 128, 0, st>>>(g.nx, g.ny, user);
  if (g.cyclic_y) k_setcyclic_user_y<<<nblk(g.nx + 4, 128), 128, 0, st>>>(g.nx, g.ny, user);
}

__global__ void k_fill_pseudorandom(double* __restrict__ a, size_t n, uint32_t seed) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    // 32-bit integer mix of (k, seed); the top 31 bits give a uniform value in [-1, 1)
    uint32_t h = (uint32_t)k * 0x9E3779B1u ^ seed;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    a[k] = (double)(h >> 1) * (2.0 / 2147483648.0) - 1.0;
  }
}

void launch_fill_pseudorandom(double* a, size_t n, uint32_t seed, cudaStream_t st) {
  k_fill_pseudorandom<<<std::min<size_t>(nblk(n, 256), 4096), 256, 0, st>>>(a, n, seed);
}

void launch_to_f32(const double* a, float* b, size_t n, cudaStream_t st) {
  k_to_f32<<<std::min<size_t>(nblk(n, 256), 4096), 256, 0, st>>>(a, b, n);
}

void launch_residual_f32(const Geo& g, const OpDev<double>& op, const double* forc_user, const double* x, double s,
                         float* b32, cudaStream_t st) {
  k_residual_f32<<<nblk(full_count(g), 256), 256, 0, st>>>(g, op, forc_user, x, s, b32);
}

void launch_add_correction(const Geo& g, double* x, const float* e, double c, cudaStream_t st) {
  k_add_correction<<<std::min<size_t>(nblk((size_t)g.nx * g.ny, 256), 4096), 256, 0, st>>>(g, x, e, c);
}

void launch_fill_cyclic(const Geo& g, double* a, cudaStream_t st) {
  if (g.cyclic_x || g.cyclic_y) k_fill_cyclic_padded<<<nblk(full_count(g), 256), 256, 0, st>>>(g, a);
}

void launch_apply_op_user(const Geo& g, const OpDev<double>& op, const double* p_user, double* res_user,
                          double* scratch, cudaStream_t st) {
  launch_pack(g, p_user, scratch, false, st);
  const size_t n = full_count(g);
  k_apply_user<<<nblk(n, 256), 256, 0, st>>>(g, op, scratch, res_user);
}

void launch_line_integral_uv(int nx, const IslandDev& isl, const LineGeo& lg, const double* u, const double* v,
                             int k0, int nk, double* out, cudaStream_t st) {
  if (nk <= 0) return;
  k_line_uv<<<nk, kLineThreads, 0, st>>>(nx, isl, lg, u, v, k0, out);
}

void launch_line_integral_psi(int nx, int ny, const IslandDev& isl, const LineGeo& lg, const double* psi,
                              size_t stride, int nfields, int k0, int nk, double* out, cudaStream_t st) {
  (void)ny;
  if (nk <= 0 || nfields <= 0) return;
  k_line_psi<<<dim3(nk, nfields), kLineThreads, 0, st>>>(nx, isl, lg, psi, stride, k0, nk, out);
}

void launch_island_solve(int nisle, const double* lu, const int* ipiv, const double* lf, const double* lp,
                         double* dpsin, int tau, cudaStream_t st) {
  if (nisle <= 1) return;
  k_island_solve<<<1, 32, sizeof(double) * (nisle - 1), st>>>(nisle, lu, ipiv, lf, lp, dpsin, tau);
}

void launch_hydrostatic(const StepDev& s, cudaStream_t st) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  k_hydrostatic<<<nblk(n2, 256), 256, 0, st>>>(s);
}

void launch_sf_forcing(const StepDev& s, double* fpx, double* fpy, double* forc, cudaStream_t st) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  k_sf_columns<<<nblk(n2, 128), 128, 0, st>>>(s, fpx, fpy);
  Geo g{s.nx, s.ny, 0, s.cyclic_x, s.cyclic_y};
  launch_setcyclic_user(g, fpx, st);
  launch_setcyclic_user(g, fpy, st);
  k_sf_forc<<<nblk(n2, 256), 256, 0, st>>>(s, fpx, fpy, forc);
}

void launch_first_guess(const Geo& g, double* a1, const double* a0, const double* am, cudaStream_t st) {
  const size_t n2 = full_count(g);
  k_first_guess<<<nblk(n2, 256), 256, 0, st>>>(n2, a1, a0, am);
}

void launch_sf_psi_update(const StepDev& s, const double* psin, int nisle, const double* dpsin, cudaStream_t st) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  k_sf_psi<<<nblk(n2, 256), 256, 0, st>>>(s, psin, nisle, dpsin);
}

void launch_sf_velocity_update(const StepDev& s, cudaStream_t st) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  k_sf_velocity<<<nblk(n2, 128), 128, 0, st>>>(s);
}

void launch_sp_forcing(const StepDev& s, int free_surface, double* fpx, double* fpy, double* forc, cudaStream_t st) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  k_sp_columns<<<nblk(n2, 128), 128, 0, st>>>(s, fpx, fpy);
  Geo g{s.nx, s.ny, 0, s.cyclic_x, s.cyclic_y};
  launch_setcyclic_user(g, fpx, st);
  launch_setcyclic_user(g, fpy, st);
  k_sp_forc<<<nblk(n2, 256), 256, 0, st>>>(s, free_surface, fpx, fpy, forc);
}

void launch_residual(const Geo& g, const OpDev<double>& op, const double* forc_user, const double* sol_padded,
                     double* part, int nb, double* out2, cudaStream_t st) {
  k_residual<<<nb, 256, 0, st>>>(g, op, forc_user, sol_padded, part);
  k_residual_final<<<1, 32, 0, st>>>(part, nb, out2);
}

void launch_sp_velocity_update(const StepDev& s, cudaStream_t st) {
  const size_t n2 = (size_t)(s.nx + 4) * (s.ny + 4);
  k_sp_velocity<<<nblk(n2, 128), 128, 0, st>>>(s);
}

}  // namespace pyomgpu
