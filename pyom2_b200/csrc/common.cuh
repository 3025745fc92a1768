// Device-side building blocks shared by the external-mode kernels.
//
// * Padded field layout: a 2-D field of the pyOM2 grid (Fortran extents
//   (1-onx:nx+onx, 1-onx:ny+onx), onx = 2, main_module.f90:35) is stored with
//   a row pitch that is a multiple of 32 elements and an x offset that puts the
//   first interior column (Fortran i = 1) on a 32-byte boundary, so every
//   warp-wide row access of the interior starts on a DRAM sector.
// * A software grid barrier for persistent cooperative kernels whose waits are
//   bounded by %globaltimer: on time-out the kernel records PYOMGPU_TIMEOUT and
//   returns instead of spinning forever.
// * Deterministic grid reductions: every block publishes its partials to a
//   slot, and after the barrier every block sums all slots in the same fixed
//   order, so all blocks obtain bit-identical scalars and take identical
//   branch decisions (the role of MPI_Allreduce in parallel_mpi.f90:232-277).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pyomgpu.h"

namespace pyomgpu {

constexpr int kOnx = 2;
constexpr int kXOff = 2;  // Fortran i = -1 sits at element kXOff

struct Geo {
  int nx, ny;        // interior points
  int pitch;         // elements per stored row
  int cyclic_x, cyclic_y;
  __host__ __device__ __forceinline__ size_t at(int i, int j) const {
    return (size_t)(j + 1) * (size_t)pitch + (size_t)(i + 1 + kXOff);
  }
  __host__ __device__ __forceinline__ size_t size() const { return (size_t)(ny + 2 * kOnx) * (size_t)pitch; }
};

// Fortran-layout (ld = nx+4) offset of (i,j), as f2py hands the arrays over.
__host__ __device__ __forceinline__ size_t fidx(int nx, int i, int j) {
  return (size_t)(i + 1) + (size_t)(j + 1) * (size_t)(nx + 2 * kOnx);
}

// Halo positions that setcyclic_xy (parallel_none.f90:188-211) fills from the
// interior point (i,j): at most one x copy and one y copy (nx, ny >= 4).
__device__ __forceinline__ void cyclic_copies(const Geo& g, int i, int j, int& xc, int& yc) {
  xc = 0x7fffffff;
  yc = 0x7fffffff;
  if (g.cyclic_x) xc = (i <= kOnx) ? i + g.nx : ((i > g.nx - kOnx) ? i - g.nx : xc);
  if (g.cyclic_y) yc = (j <= kOnx) ? j + g.ny : ((j > g.ny - kOnx) ? j - g.ny : yc);
}

// Store v at interior (i,j) and at every halo position that setcyclic_xy
// would fill with it.
template <typename T>
__device__ __forceinline__ void store_cyclic(T* __restrict__ a, const Geo& g, int i, int j, T v) {
  a[g.at(i, j)] = v;
  int xc, yc;
  cyclic_copies(g, i, j, xc, yc);
  if (xc != 0x7fffffff) a[g.at(xc, j)] = v;
  if (yc != 0x7fffffff) {
    a[g.at(i, yc)] = v;
    if (xc != 0x7fffffff) a[g.at(xc, yc)] = v;
  }
}

// a += d at interior (i,j) and at its setcyclic_xy copies.
template <typename T>
__device__ __forceinline__ void add_cyclic(T* __restrict__ a, const Geo& g, int i, int j, T d) {
  a[g.at(i, j)] += d;
  int xc, yc;
  cyclic_copies(g, i, j, xc, yc);
  if (xc != 0x7fffffff) a[g.at(xc, j)] += d;
  if (yc != 0x7fffffff) {
    a[g.at(i, yc)] += d;
    if (xc != 0x7fffffff) a[g.at(xc, yc)] += d;
  }
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Control block in device memory shared by the blocks of one persistent launch.
struct SyncCtl {
  unsigned long long arrive;  // monotonically increasing arrival count (reset per launch)
  int error;                  // PYOMGPU_TIMEOUT once any block gave up waiting
  int pad;
};

// Block-wide barrier across the whole grid.  Returns false on time-out (or when
// another block already timed out); the caller must then leave the kernel.
__device__ __forceinline__ bool grid_sync(SyncCtl* ctl, unsigned nblocks, unsigned long long& epoch,
                                          unsigned long long timeout_ns, unsigned extra = 0) {
  __shared__ int s_ok;
  __syncthreads();
  epoch += 1;  // every thread keeps the same count (slot parities derive from it)
  if (threadIdx.x == 0) {
    const unsigned long long target = epoch * (unsigned long long)nblocks + extra;
    red_release_add_u64(&ctl->arrive, 1ull);
    int ok = 1;
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    while (ld_acquire_u64(&ctl->arrive) < target) {
      if ((++spins & 63u) == 0u) {
        if (ld_relaxed_i32(&ctl->error) != 0) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > timeout_ns) {
          atomicExch(&ctl->error, PYOMGPU_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---------------------------------------------------------------------------
// deterministic reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, m));
  return v;
}

// Reduce NV values per thread over the block (sums, except index kMaxSlot
// which is a max when >= 0); thread 0 gets the result in out[].  Fixed order.
template <int NV, int kMaxSlot, int kThreads>
__device__ __forceinline__ void block_reduce(const double (&v)[NV], double (&out)[NV]) {
  __shared__ double sh[kThreads / 32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double r = (k == kMaxSlot) ? warp_max(v[k]) : warp_sum(v[k]);
    if (lane == 0) sh[w][k] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double r = sh[0][k];
      for (int q = 1; q < kThreads / 32; q++) r = (k == kMaxSlot) ? fmax(r, sh[q][k]) : r + sh[q][k];
      out[k] = r;
    }
  }
  __syncthreads();
}

// After a grid_sync: every block combines all published partials
// (slots[b*stride + k], b < nblocks) with every thread loading at most a few
// slots at once (one L2 round trip), then a fixed-order block reduction, so all
// blocks obtain the same values.  Slot kMaxSlot (if >= 0) is a max, the others
// sums.  Result broadcast to every thread.
template <int NV, int kMaxSlot, int kThreads>
__device__ __forceinline__ void grid_collect(const double* __restrict__ slots, int stride, unsigned nblocks,
                                             double (&out)[NV]) {
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = 0.0;
  constexpr int kMaxPer = 4;  // nblocks <= 4 * kThreads
#pragma unroll
  for (int u = 0; u < kMaxPer; u++) {
    const unsigned b = threadIdx.x + u * kThreads;
    if (b < nblocks) {
#pragma unroll
      for (int k = 0; k < NV; k++) {
        const double x = __ldcg(slots + (size_t)b * stride + k);
        v[k] = (k == kMaxSlot) ? fmax(v[k], x) : v[k] + x;
      }
    }
  }
  __shared__ double sh_out[NV];
  double r[NV];
  block_reduce<NV, kMaxSlot, kThreads>(v, r);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) sh_out[k] = r[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) out[k] = sh_out[k];
  __syncthreads();
}

// After a grid_sync: every block sums all published slots (layout
// slots[block*NV + k]) in a fixed order; warp 0 does the work, the result is
// broadcast through shared memory.
template <int NV, int kMaxSlot>
__device__ __forceinline__ void grid_allreduce(const double* __restrict__ slots, unsigned nblocks, double (&out)[NV]) {
  __shared__ double sh[NV];
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double r = (k == kMaxSlot) ? 0.0 : 0.0;
      for (unsigned b = lane; b < nblocks; b += 32) {
        double x = __ldcg(slots + (size_t)b * NV + k);
        r = (k == kMaxSlot) ? fmax(r, x) : r + x;
      }
      r = (k == kMaxSlot) ? warp_max(r) : warp_sum(r);
      if (lane == 0) sh[k] = r;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) out[k] = sh[k];
  __syncthreads();
}

}  // namespace pyomgpu
