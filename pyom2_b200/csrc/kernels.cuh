// Host-callable launchers of the non-CG kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "ops.cuh"

namespace pyomgpu {

// Geometry inputs on the device (Fortran layout, ld nx+4) used while building operators.
struct GridDev {
  int nx, ny;
  const double *dxt, *dxu, *dyt, *dyu, *cost, *cosu;  // 1-D, length nx+4 / ny+4
  const double *hur, *hvr, *hu, *hv, *maskT_top;      // Fortran layout
};

struct OpBuf {
  double *FX = nullptr, *FY = nullptr, *W = nullptr;  // padded
  double *ax = nullptr, *bx = nullptr, *by = nullptr; // 1-D
  double dcoef = 0.0;
  OpDev<double> dev() const { return OpDev<double>{FX, FY, ax, bx, by, W, dcoef}; }
};

void launch_build_op_streamfunction(const GridDev& gd, const Geo& g, OpBuf& op, cudaStream_t st);
void launch_build_op_surf_press(const GridDev& gd, const Geo& g, OpBuf& op, cudaStream_t st);
// Z = 1/diag (0 where diag = 0), zero at the given interior points, cyclic halo copies.
void launch_build_inv_diag(const Geo& g, OpBuf& op, const int* bnd_i, const int* bnd_j, int nbnd, cudaStream_t st);

// user (Fortran, ld nx+4) <-> padded
void launch_pack(const Geo& g, const double* user, double* padded, bool setcyclic, cudaStream_t st);
void launch_unpack(const Geo& g, const double* padded, double* user, bool setcyclic, bool interior_only,
                   bool zero_halo, cudaStream_t st);
void launch_setcyclic_user(const Geo& g, double* user, cudaStream_t st);
// setcyclic_xy on a padded field
void launch_fill_cyclic(const Geo& g, double* padded, cudaStream_t st);

// res = A p over the interior, zero halo; p and res in Fortran layout.
void launch_apply_op_user(const Geo& g, const OpDev<double>& op, const double* p_user, double* res_user,
                          double* scratch_padded, cudaStream_t st);

// Island line integrals.  Segments of every island's perimeter are listed as
// (i, j, dir) with dir in {0:E,1:W,2:N,3:S}, offsets per island in seg_off.
struct IslandDev {
  int nisle = 0;
  int* seg_i = nullptr;
  int* seg_j = nullptr;
  int* seg_d = nullptr;
  int* seg_off = nullptr;  // nisle + 1
};
struct LineGeo {
  const double *dxu, *dyu, *cost, *cosu, *dxt, *dyt;  // 1-D
  const double *hur, *hvr, *maskU_top, *maskV_top;      // Fortran layout
};
// out[q*nisle_used + k] for q over fields, k islands [k0, k0+nk): integral of (u,v) given as arrays.
void launch_line_integral_uv(int nx, const IslandDev& isl, const LineGeo& lg, const double* u, const double* v,
                             int k0, int nk, double* out, cudaStream_t st);
// integrals of the velocity of streamfunction fields psi[f] (Fortran layout, stride n2 between
// fields): out[f*nk + k]
void launch_line_integral_psi(int nx, int ny, const IslandDev& isl, const LineGeo& lg, const double* psi,
                              size_t field_stride, int nfields, int k0, int nk, double* out, cudaStream_t st);

// Solve line_psin(2:,2:) x = rhs(2:) - psi0(2:) with the LU factors computed on the
// host (DGESV pivoting); writes dpsin(2:nisle, tau).
void launch_island_solve(int nisle, const double* lu, const int* ipiv, const double* line_forc,
                         const double* line_psi0, double* dpsin, int tau, cudaStream_t st);

// out2[0] = sum (forc - A sol)^2, out2[1] = sum forc^2 over points with W != 0.
// part needs 2*nb doubles.
void launch_residual(const Geo& g, const OpDev<double>& op, const double* forc_user, const double* sol_padded,
                     double* part, int nb, double* out2, cudaStream_t st);

// a[k] = a deterministic pseudo-random value in [-1, 1) (integer hash of k and seed)
void launch_fill_pseudorandom(double* a, size_t n, uint32_t seed, cudaStream_t st);

// mixed precision helpers
void launch_to_f32(const double* a, float* b, size_t n, cudaStream_t st);
// b32 = s (forc - A x) at the unknowns (W != 0), zero elsewhere (x padded with valid halo)
void launch_residual_f32(const Geo& g, const OpDev<double>& op, const double* forc_user, const double* x, double s,
                         float* b32, cudaStream_t st);
// x += c e over the interior
void launch_add_correction(const Geo& g, double* x, const float* e, double c, cudaStream_t st);

// ---- solve_streamfunction / solve_pressure pre and post ----------------------
struct StepDev {
  int nx, ny, nz, cyclic_x, cyclic_y;
  int taum1, tau, taup1;
  double dt_mom, AB_eps, grav, rho_0;
  const double *dxt, *dxu, *dyt, *dyu, *cost, *cosu, *dzt, *dzw;
  const double *hur, *hvr;
  const double *maskT, *maskU, *maskV, *rho, *du_mix, *dv_mix;
  double *u, *v, *du, *dv, *p_hydro, *psi, *dpsi;
};
void launch_hydrostatic(const StepDev& s, cudaStream_t st);
// streamfunction: du/dv gradient, fpx/fpy = sum (du+du_mix) maskU dzt * hur (full array), setcyclic
void launch_sf_forcing(const StepDev& s, double* fpx, double* fpy, double* forc, cudaStream_t st);
void launch_first_guess(const Geo& g, double* a_taup1, const double* a_tau, const double* a_taum1, cudaStream_t st);
void launch_sf_psi_update(const StepDev& s, const double* psin, int nisle, const double* dpsin, cudaStream_t st);
void launch_sf_velocity_update(const StepDev& s, cudaStream_t st);
// surface pressure
void launch_sp_forcing(const StepDev& s, int free_surface, double* fpx, double* fpy, double* forc, cudaStream_t st);
void launch_sp_velocity_update(const StepDev& s, cudaStream_t st);

}  // namespace pyomgpu
