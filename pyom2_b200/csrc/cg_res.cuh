// Parameters of the on-chip-resident Jacobi-PCG kernel (cg_res.cu): one
// block per SM owns one rectangular piece of the grid for the whole solve.
#pragma once
#include "cg_ref.cuh"

namespace pyomgpu {

constexpr int kResThreads = 512;
constexpr int kResWorkers = kResThreads - 32;  // warps 1-15 own the points; warp 0 runs the reductions
constexpr int kResMaxSlots = 160;              // reduction slots warp 0 polls (blocks + 1)
constexpr int kResSlotWords = 8;               // words per reduction slot (at most 7 partial sums)
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
  double* hx;          // halo exchange: a 4-word record per padded position, (Z*res, direction) for
                       // the two-reduction kernel, (res, A Z res, A p) in two alternating buffers
                       // (8 words per position) for the single-reduction one
  long long hsize;     // padded positions (records)
  double* slots;       // 4 x nslot x kResSlotWords words: 3 rotating buffers of kResSlotWords words per
                       // block (single-reduction kernel; all empty on entry), or 2 buffers of
                       // 2 kResSlotWords tagged words per block (two-reduction kernel)
  int nslot;           // gridDim.x + 1
  int npx, npy;        // pieces in x and y (gridDim.x = npx * npy)
  int wmax, hmax;      // largest piece extents: shared-memory layout and thread columns
  double eps;
  double rtol;
  int max_it;
  SyncCtl* ctl;
  unsigned long long timeout_ns;
  unsigned stall_extra;  // test hook: the first reduction also awaits a slot nobody writes
  int weighted;          // multi-solve kernel: inner products weighted by the cell area D = 1/(ax by)
  unsigned tag_gen;      // 0 .. 4094, different for consecutive solves of a context: the high bits of
                         // the epoch tags of the two-reduction kernel's slots and exchange records
  CGResult* out;
  // phase timestamps of the traced instantiation (cg_res_kernel<P, true>):
  // %globaltimer at kResTracePhases points of loop trips trace_it0 ..
  // trace_it0 + trace_nit - 1, per block: trace[(block * trace_nit + trip -
  // trace_it0) * kResTracePhases + phase]
  unsigned long long* trace;
  int trace_it0, trace_nit;
  // FP32 fields (cg_res32_kernel): operator copy, right-hand side, solution and
  // residual, all in the padded layout; the exchange records then hold two
  // tagged words per position
  OpDev<float> op32;
  const float* forc32;
  float* sol32;
  float* res32;
};

// Many resident solves in one launch (cg_res_multi_kernel), scheduled on the
// host: every block runs its own list of (job, piece) entries in order; the
// blocks of one job (its gang) meet at the job's join counter before they
// start it.  Every job has its own CGResParams, slots, exchange records
// (tagged), error flag and result.  The lists are ordered by planned start
// time, one total order for all blocks, so no set of gangs can wait on one
// another in a cycle.
struct ResMultiParams {
  const CGResParams* jobs;
  const int* list_off;   // gridDim.x + 1 offsets into list
  const int2* list;      // (job, piece index within the job)
  int* join;             // per job, blocks arrived (zero on entry)
  unsigned long long* times;  // per job: %globaltimer when its gang has assembled and when piece 0 ends
  int* error;            // PYOMGPU_TIMEOUT when a gang did not assemble within gang_timeout_ns
  unsigned long long gang_timeout_ns;
};

// Phases of the trace (worker warp 1 lane 0 unless noted "ctl": warp 0 lane 0):
//  0 sweep A start, 1 direction in shared memory (workers' barrier), 2 stencil
//  and partials done, 3 after S1, 4 after S2 (alpha known), 5 residual updated
//  and boundary staged, 6 exchange records written, 7 after S1, 8 solution
//  updated, 9 after S2 (halo loaded, beta known); ctl: 10 after S1 (A), 11 slot
//  published, 12 all slots acquired, 13 control step done, 14 after S1 (B),
//  15 slot published, 16 all slots acquired, 17 control step done.
constexpr int kResTracePhases = 18;

// Dynamic shared memory of a w x h piece (the larger of the two kernels'
// needs): the stencil operand with its one-cell halo, the x- and y-face
// couplings, the row factors bx, by, the staged boundary values (up to 3 per
// boundary entry) and the received halo records (4 words each, 16-byte
// aligned, single-reduction kernel).
__host__ __device__ constexpr size_t res_smem_bytes(int w, int h) {
  return 8 * ((((size_t)(w + 2) * (h + 2) + (size_t)(w + 1) * h + (size_t)w * (h + 1) + 2 * (size_t)h +
                6 * (size_t)(w + h)) + 1) / 2 * 2 + 8 * (size_t)(w + h));
}

// Threads that a w x h piece needs with p points per thread.
__host__ __device__ constexpr int res_threads(int w, int h, int p) { return w * ((h + p - 1) / p); }

// The resident kernel for p points per thread: two reductions per iteration
// (the reference's recurrences) or one (single = true: A p by recurrence and
// (p, Ap) by its exact expansion in products of the sweep before).
const void* cg_res_kernel_ptr(int p, bool single);
// The two-reduction kernel with FP32 fields at p = 16 or 32 points per thread.
const void* cg_res32_kernel_ptr(int p);
// Dynamic shared memory of a w x h piece of the FP32 kernel: the stencil
// operand with its halo, FX, FY, bx, by and the staged boundary values.
__host__ __device__ constexpr size_t res32_smem_bytes(int w, int h) {
  return 4 * (((size_t)(w + 2) * (h + 2) + (size_t)(w + 1) * h + (size_t)w * (h + 1) + 2 * (size_t)h +
               4 * (size_t)(w + h) + 3) / 4 * 4);
}
// The multi-solve launch of the two-reduction kernel at 16 points per thread
// (weighted: all its solves take the area-weighted products).
const void* cg_res_multi_kernel_ptr(bool weighted = false);
// The traced instantiation of the two-reduction kernel (same arithmetic).
const void* cg_res_trace_kernel_ptr(int p);

}  // namespace pyomgpu
