// Parameters of the persistent reference-algorithm CG kernels (cg_ref.cu).
#pragma once
#include "common.cuh"
#include "ops.cuh"

namespace pyomgpu {

constexpr int kCGThreads = 256;

struct CGResult {
  int iterations;
  int converged;
  int status;
  int pad;
  double est;
};

struct CGRefParams {
  Geo g;
  OpDev<double> op;
  const double* forc;  // Fortran layout (ld nx+4), device
  double* sol;         // padded; streamfunction: sol, surf_press: psi(:,:,taup1)
  double* res;         // padded
  double* s[2];        // padded, double-buffered search direction (zero halos)
  double* As;          // padded
  double eps;          // congr_epsilon
  int max_it;          // congr_max_iterations
  double rtol;         // > 0: extra stop on ||res||/||forc|| over the unknowns
  int R, SX, SY;       // strip rows, strips in x and y
  SyncCtl* ctl;
  double* slots;       // 2 * gridDim.x * 4 doubles
  unsigned long long timeout_ns;
  unsigned stall_extra;  // test hook: first barrier waits for this many extra blocks
  CGResult* out;
};

const void* cg_ref_kernel_ptr(bool surf_press);

}  // namespace pyomgpu
