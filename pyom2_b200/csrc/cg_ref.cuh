// Parameters of the persistent reference-algorithm CG kernels (cg_ref.cu).
#pragma once
#include <cuda.h>

#include "common.cuh"
#include "ops.cuh"
#include "tma.cuh"

namespace pyomgpu {

constexpr int kCGThreads = 256;
// shared memory: five kBoxX x kBoxY FP64 tiles (128-byte aligned) + the mbarrier
constexpr size_t kTileBytes = ((size_t)kBoxX * kBoxY * 8 + 127) / 128 * 128;
constexpr size_t kCGSmem = 5 * kTileBytes + 128;

struct CGResult {
  int iterations;
  int converged;
  int status;
  int pad;
  double est;
};

struct alignas(64) CGRefParams {
  // tensor maps of the fields the stencil sweep stages through shared memory
  CUtensorMap map_res, map_W, map_FX, map_FY, map_s[2];
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
  int ntx, nty;        // tiles in x and y (kTileX x kTileY interior points each)
  SyncCtl* ctl;
  double* slots;       // 2 * gridDim.x * 4 doubles
  unsigned long long timeout_ns;
  unsigned stall_extra;  // test hook: first barrier waits for this many extra blocks
  CGResult* out;
};

const void* cg_ref_kernel_ptr(bool surf_press);

}  // namespace pyomgpu
