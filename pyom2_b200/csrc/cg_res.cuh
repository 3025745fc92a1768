// Parameters of the on-chip-resident Jacobi-PCG kernel (cg_res.cu): one
// block per SM owns one rectangular piece of the grid for the whole solve.
#pragma once
#include "cg_ref.cuh"

namespace pyomgpu {

constexpr int kResThreads = 512;
constexpr int kResWorkers = kResThreads - 32;  // warps 1-15 own the points; warp 0 runs the reductions
constexpr int kResMaxSlots = 160;              // reduction slots warp 0 polls (blocks + 1)
// Points per thread along a column segment (template instances of the kernel).
constexpr int kResP[] = {4, 8, 16};
constexpr int kResNP = 3;

// Empty-slot pattern of the reduction words: all bits set
// (a NaN no arithmetic result is written as; cudaMemset(0xFF) fills it).
constexpr unsigned long long kResEmpty = 0xFFFFFFFFFFFFFFFFull;

struct CGResParams {
  Geo g;
  OpDev<double> op;    // FX, FY, ax, bx, by, W = Z
  const double* forc;  // Fortran layout (ld nx+4), device
  double* sol;         // padded, halo valid on entry; interior updated
  double* res;         // padded; the residual of the last iterate on exit (with setcyclic copies)
  double* hx;          // halo exchange: a 4-word record per padded position (Z*res, direction)
  long long hsize;     // padded positions (records)
  double* slots;       // 3 buffers x nslot x 4 reduction words, all empty on entry
  int nslot;           // gridDim.x + 1
  int npx, npy;        // pieces in x and y (gridDim.x = npx * npy)
  int wmax, hmax;      // largest piece extents: shared-memory layout and thread columns
  double eps;
  double rtol;
  int max_it;
  SyncCtl* ctl;
  unsigned long long timeout_ns;
  unsigned stall_extra;  // test hook: the first reduction also awaits a slot nobody writes
  CGResult* out;
};

// Dynamic shared memory of a w x h piece: the direction with its one-cell
// halo, the x- and y-face couplings, the row factors bx, by and the staged
// boundary values (2 per boundary entry).
__host__ __device__ constexpr size_t res_smem_bytes(int w, int h) {
  return 8 * ((size_t)(w + 2) * (h + 2) + (size_t)(w + 1) * h + (size_t)w * (h + 1) + 2 * (size_t)h +
              4 * (size_t)(w + h));
}

// Threads that a w x h piece needs with p points per thread.
__host__ __device__ constexpr int res_threads(int w, int h, int p) { return w * ((h + p - 1) / p); }

const void* cg_res_kernel_ptr(int p);

}  // namespace pyomgpu
