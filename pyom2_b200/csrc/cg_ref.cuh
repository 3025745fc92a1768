// Parameters of the persistent reference-algorithm CG kernels (cg_ref.cu).
#pragma once
#include <cuda.h>

#include "common.cuh"
#include "ops.cuh"
#include "tma.cuh"

namespace pyomgpu {

constexpr int kCGThreads = 256;
// Tile shape is a launch parameter (tx x ty interior points, box (tx+4) x
// (ty+2)); tx even so every box starts on a 16-byte boundary.  Shared memory:
// five boxes (128-byte aligned) + the mbarrier.
constexpr int kCGMaxTX = 128, kCGMaxTY = 32;
__host__ __device__ constexpr size_t cg_box_bytes(int tx, int ty) {
  return ((size_t)(tx + 4) * (ty + 2) * 8 + 127) / 128 * 128;
}
__host__ __device__ constexpr size_t cg_smem_bytes(int tx, int ty) { return 5 * cg_box_bytes(tx, ty) + 128; }
constexpr size_t kCGSmem = cg_smem_bytes(kTileX, kTileY);        // default tile
constexpr size_t kCGSmemMax = cg_smem_bytes(kCGMaxTX, kCGMaxTY);  // attribute reserved once

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
  int tx, ty;          // tile shape (interior points)
  int ntx, nty;        // tiles in x and y
  SyncCtl* ctl;
  double* slots;       // 2 * gridDim.x * 4 doubles
  unsigned long long timeout_ns;
  unsigned stall_extra;  // test hook: first barrier waits for this many extra blocks
  CGResult* out;
};

const void* cg_ref_kernel_ptr(bool surf_press);

}  // namespace pyomgpu
