// Parameters of the pipelined single-sweep PCG kernel (cg_pipe.cu).
#pragma once
#include <cuda.h>

#include "common.cuh"
#include "ops.cuh"
#include "tma.cuh"

namespace pyomgpu {

constexpr int kPipeThreads = 256;

struct PipeResult {
  int iterations;
  int status;
  double rr;  // ||r||^2 over the unknowns at exit (recursive residual)
  double bb;  // ||b||^2 over the unknowns
};

template <typename T>
struct alignas(64) PipeParams {
  CUtensorMap map_r[2], map_A[2], map_s[2], map_Z, map_FX, map_FY;
  Geo g;
  OpDev<T> op;       // W = Jacobi inverse Z (0 on Dirichlet points)
  const T* b;        // right-hand side, padded
  T* x;              // in/out, padded (own points updated; halo valid on entry)
  T* r[2];           // double-buffered residual, zero halos, cyclic copies written by owners
  T* A[2];           // double-buffered A s
  T* s[2];           // double-buffered search direction
  double rtol;       // stop when ||r|| <= rtol ||b|| over the unknowns
  int max_it;
  int ntx, nty;      // kTileX x kTileY tiles
  SyncCtl* ctl;
  double* slots;     // 2 * gridDim.x * 8
  unsigned long long timeout_ns;
  PipeResult* out;
};

const void* cg_pipe_kernel_ptr(bool f32);
size_t pipe_smem_bytes(bool f32);
// fills the tensor maps of P from its pointers; 0 on success
template <typename T>
int pipe_encode_all(PipeParams<T>& P);

}  // namespace pyomgpu
