// Persistent work-queue kernel: many independent congrad_streamfunction solves
// (the island right-hand sides of streamfunction_init, or unevenly sized grids)
// in one launch (cg_batch.cu).
#pragma once
#include "common.cuh"
#include "ops.cuh"

namespace pyomgpu {

constexpr int kBatchThreads = 256;

// One solve: grid, operator and work buffers (constant during a launch).
struct BatchProblem {
  Geo g;
  OpDev<double> op;    // FX, FY, ax, bx, by, W = Z
  const double* forc;  // Fortran layout (ld nx+4)
  double* sol;         // padded, halo set (setcyclic) on entry
  double* res;         // padded work buffers, zero on entry
  double* s[2];
  double* As;
  double eps;
  double rtol;         // > 0: extra stop on ||res|| / ||forc|| over the unknowns (||res|| / ||res_0||
                       // for a zero forcing, e.g. the psin solves)
  int max_it;
  int weighted;        // 1: inner products weighted by the cell area D = 1/(ax by) = dxu dyu cosu, in
                       // which A = D^-1 S is self-adjoint (exact Jacobi-PCG on the symmetric S); 0: the
                       // reference's Euclidean products
  int tile0, ntx, nty; // first task index, tiles in x and y
};

// Scalars of one solve, advanced only by the block that reduces at a grid
// barrier and read by all blocks through L2 (11 x 8 bytes).
struct BatchState {
  int n, phase;  // iteration; phase: 0 done, 1 sweep A next, 2 sweep B next
  int status, converged, stop_after, pad;
  double beta, betam1, betamin, step1, est, bq, alpha, bb;
};
static_assert(sizeof(BatchState) == 88, "BatchState is moved as 11 words");

// Most problems of one launch (their active list is kept in shared memory;
// larger batches run in several launches).
constexpr int kBatchActMax = 1024;

struct BatchParams {
  const BatchProblem* probs;
  BatchState* state;     // zero on entry
  int nprob;
  int ntasks;            // total tiles of all problems
  double* part;          // per task, 4 partials
  int* done;             // per problem, tiles finished in the current sweep (zero on entry)
  // the problems taking part in the next sweep, rebuilt at every grid barrier:
  // act_prob[0 .. act_n-1], their tiles at act_off[k] .. act_off[k+1]-1 of the
  // sweep's task range (on entry: every problem, for the initial sweep)
  int* act_n;
  int* act_prob;         // nprob
  int* act_off;          // nprob + 1
  SyncCtl* ctl;
  unsigned long long* gen;  // release flag of the block that rebuilt the list
  unsigned long long timeout_ns;
  unsigned stall_extra;  // test hook: the first barrier awaits this many blocks more than launched
};

// Cooperative launch (all blocks co-resident: grid <= occupancy x SMs).
cudaError_t launch_cg_batch(const BatchParams& P, int grid, cudaStream_t st);
const void* cg_batch_kernel_ptr();

}  // namespace pyomgpu
