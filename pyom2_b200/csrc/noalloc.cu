// Allocation-free congrad_streamfunction.
//
// Some callers cannot call cudaMalloc at all: an ocean model embedded in a
// host application that hands the GPU over with a fixed memory budget
// already claimed by its own pool allocator, code that runs while a memory
// pool forbids new device allocations, or a caller that must not touch the
// allocator from its time-stepping loop (an allocation there can synchronise
// the device or fail under memory pressure half-way through a run).  For
// them this file provides one entry point that solves with scratch memory
// the library holds itself: a file-scope __device__ array of kNoAllocBytes
// (64 MiB) on every GPU that uses it, held until the process exits.  CUDA
// loads a library's device code lazily by default, so the array (and this
// file's kernels) are materialised on the device by the first call made on
// it: make that call at set-up, while device memory is still free and before
// any stream capture.  Under memory pressure that first call can fail with
// PYOMGPU_ECUDA; later calls take no device memory.
//
// The caller passes only inputs and outputs (device pointers): the grid
// metrics and hur/hvr, the island perimeter points, forc and sol.  The
// operator, the Jacobi inverse, every work vector, the barrier control block
// and the reduction slots are placed in the static array.  Every call reuses
// that same array and finds the previous call's contents in it, so each call
// clears what must start at zero; two calls that overlap on the GPU (other
// streams, other host threads) race on it and must not be issued.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/pyomgpu.h"
#include "cg_ref.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace pyomgpu {
void set_last_error(const char* msg);  // capi.cu

namespace {

constexpr size_t kNoAllocBytes = PYOMGPU_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// In host code g_noalloc_scratch names a host-side shadow, not device memory;
// the device address comes from cudaGetSymbolAddress, once per device.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_dev[kMaxDevices] = {};

int nfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  set_last_error(buf);  // reported by pyomgpu_last_error()
  return code;
}

// Device memory of the current device, or managed memory.  Memory of another
// GPU is refused: the kernels would read it over the peer path, or fault where
// peer access is off.
bool on_device(const void* p, int dev) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
}

// Device address of the scratch array on the current device (set-up on the
// first call made on each device).
int scratch_base(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return nfail(PYOMGPU_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return nfail(PYOMGPU_EINVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return nfail(PYOMGPU_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_scratch_dev[dev] = p;
  }
  *out = g_scratch_dev[dev];
  return 0;
}

// Bump allocator over the static array (256-byte aligned pieces).
struct Carve {
  unsigned char* base;
  size_t used = 0;
  template <typename T>
  T* take(size_t n) {
    used = (used + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + used);
    used += n * sizeof(T);
    return p;
  }
};

}  // namespace
}  // namespace pyomgpu

using namespace pyomgpu;

extern "C" int32_t pyomgpu_congrad_streamfunction_noalloc(const pyomgpu_grid* gr, const int32_t* bnd_i,
                                                          const int32_t* bnd_j, int32_t nbnd, const double* forc,
                                                          double* sol, double congr_epsilon,
                                                          int32_t congr_max_iterations, pyomgpu_solve_info* info,
                                                          pyomgpu_stream stream) {
  if (!gr || !forc || !sol || nbnd < 0 || (nbnd > 0 && (!bnd_i || !bnd_j)))
    return nfail(PYOMGPU_EINVAL, "null argument");
  if (gr->onx != 2 || gr->nx < 4 || gr->ny < 4) return nfail(PYOMGPU_EINVAL, "bad grid size");
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return nfail(PYOMGPU_ECUDA, "cudaGetDevice failed");
  const void* need[] = {gr->dxt, gr->dxu, gr->dyt, gr->dyu, gr->cost, gr->cosu, gr->hur, gr->hvr, forc, sol};
  for (const void* p : need)
    if (!on_device(p, cur))
      return nfail(PYOMGPU_EINVAL, "every array must be device memory of the current device (no staging here)");
  if (nbnd > 0 && (!on_device(bnd_i, cur) || !on_device(bnd_j, cur)))
    return nfail(PYOMGPU_EINVAL, "island points must be device memory of the current device");
  cudaStream_t st = (cudaStream_t)stream;

  Geo g{};
  g.nx = gr->nx;
  g.ny = gr->ny;
  g.pitch = ((g.nx + 4 + kXOff) + 31) / 32 * 32;
  g.cyclic_x = gr->enable_cyclic_x ? 1 : 0;
  g.cyclic_y = gr->enable_cyclic_y ? 1 : 0;
  const size_t P = g.size();

  // launch shape: the same rule as the context path, so results match it bit for bit
  int dev = 0, nsm = 0, o1 = 0, o2 = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) ||
      cudaFuncSetAttribute(cg_ref_kernel_ptr(false), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCGSmemMax) ||
      cudaFuncSetAttribute(cg_ref_kernel_ptr(true), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCGSmemMax) ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, cg_ref_kernel_ptr(false), kCGThreads, kCGSmem) ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, cg_ref_kernel_ptr(true), kCGThreads, kCGSmem) || o1 < 1)
    return nfail(PYOMGPU_ECUDA, "device query failed");
  const int max_blocks = std::min(o1, std::max(1, o2)) * nsm;

  const size_t bytes = 8 * P * sizeof(double) + 3 * (size_t)(std::max(g.nx, g.ny) + 4) * sizeof(double) +
                       (size_t)2 * max_blocks * 4 * sizeof(double) + sizeof(SyncCtl) + sizeof(CGResult) + 16 * 256;
  if (bytes > kNoAllocBytes)
    return nfail(PYOMGPU_EINVAL,
                 "grid %dx%d needs %zu bytes of scratch, the allocation-free entry point has %zu "
                 "(about 1.0e6 padded points); use pyomgpu_congrad_streamfunction",
                 g.nx, g.ny, bytes, kNoAllocBytes);

  void* base = nullptr;
  if (int rc = scratch_base(&base)) return rc;
  Carve c{reinterpret_cast<unsigned char*>(base)};
  OpBuf op;
  op.FX = c.take<double>(P);
  op.FY = c.take<double>(P);
  op.W = c.take<double>(P);
  op.ax = c.take<double>((size_t)g.nx + 4);
  op.bx = c.take<double>((size_t)g.ny + 4);
  op.by = c.take<double>((size_t)g.ny + 4);
  double* res = c.take<double>(P);
  double* s0 = c.take<double>(P);
  double* s1 = c.take<double>(P);
  double* As = c.take<double>(P);
  double* spad = c.take<double>(P);
  double* slots = c.take<double>((size_t)2 * max_blocks * 4);
  SyncCtl* ctl = c.take<SyncCtl>(1);
  CGResult* result = c.take<CGResult>(1);

  // everything that must start at zero (the array keeps the last call's contents)
  cudaError_t e = cudaSuccess;
  for (double* p : {op.FX, op.FY, res, s0, s1})
    if (e == cudaSuccess) e = cudaMemsetAsync(p, 0, P * sizeof(double), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctl, 0, sizeof(SyncCtl), st);
  if (e != cudaSuccess) return nfail(PYOMGPU_ECUDA, "memset: %s", cudaGetErrorString(e));

  GridDev gd{g.nx, g.ny, gr->dxt, gr->dxu, gr->dyt, gr->dyu, gr->cost, gr->cosu, gr->hur, gr->hvr,
             nullptr, nullptr, nullptr};
  launch_build_op_streamfunction(gd, g, op, st);
  launch_build_inv_diag(g, op, bnd_i, bnd_j, nbnd, st);
  launch_pack(g, sol, spad, true, st);

  // the same persistent kernel as pyomgpu_congrad_streamfunction
  CGRefParams Pm{};
  if (encode_tile_map(&Pm.map_res, res, g) || encode_tile_map(&Pm.map_W, op.W, g) ||
      encode_tile_map(&Pm.map_FX, op.FX, g) || encode_tile_map(&Pm.map_FY, op.FY, g) ||
      encode_tile_map(&Pm.map_s[0], s0, g) || encode_tile_map(&Pm.map_s[1], s1, g))
    return nfail(PYOMGPU_ECUDA, "cuTensorMapEncodeTiled failed");
  Pm.tx = kTileX;
  Pm.ty = kTileY;
  Pm.ntx = (g.nx + kTileX - 1) / kTileX;
  Pm.nty = (g.ny + kTileY - 1) / kTileY;
  const int grid = std::max(1, std::min(max_blocks, Pm.ntx * Pm.nty));
  Pm.g = g;
  Pm.op = op.dev();
  Pm.forc = forc;
  Pm.sol = spad;
  Pm.res = res;
  Pm.s[0] = s0;
  Pm.s[1] = s1;
  Pm.As = As;
  Pm.eps = congr_epsilon;
  Pm.max_it = congr_max_iterations;
  Pm.rtol = 0.0;
  Pm.ctl = ctl;
  Pm.slots = slots;
  Pm.timeout_ns = 2000000000ull;
  Pm.stall_extra = 0;
  Pm.out = result;
  void* args[] = {&Pm};
  e = cudaLaunchCooperativeKernel(cg_ref_kernel_ptr(false), dim3(grid), dim3(kCGThreads), args, kCGSmem, st);
  if (e != cudaSuccess) return nfail(PYOMGPU_ECUDA, "cg launch: %s", cudaGetErrorString(e));
  launch_unpack(g, spad, sol, false, false, false, st);
  CGResult h{};
  SyncCtl hc{};
  e = cudaMemcpyAsync(&h, result, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, ctl, sizeof hc, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return nfail(PYOMGPU_ECUDA, "noalloc solve: %s", cudaGetErrorString(e));
  if (info) {
    info->iterations = h.iterations;
    info->converged = h.converged;
    info->status = hc.error ? PYOMGPU_TIMEOUT : h.status;
    info->outer_iterations = 1;
    info->estimated_error = h.est;
    info->rel_residual = -1.0;
    info->device_ms = -1.0;
    info->kernel_launches = 8;  // build x2, inverse x2-3, pack, cg, unpack
  }
  if (hc.error) return nfail(PYOMGPU_TIMEOUT, "grid barrier wait exceeded 2 s");
  return h.status;
}
