// C ABI (include/pyomgpu.h): context, island set-up and the solver entry
// points.  Host orchestration only; every array operation runs on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pyomgpu.h"
#include "cg_batch.cuh"
#include "cg_pipe.cuh"
#include "cg_ref.cuh"
#include "common.cuh"
#include "ctx.h"
#include "islands.h"
#include "kernels.cuh"

using namespace pyomgpu;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(PYOMGPU_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                                       cudaGetErrorString(e_));                                    \
  } while (0)

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) return fail(PYOMGPU_ENOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
  return 0;
}

}  // namespace

namespace pyomgpu {
// lets other translation units of the library report through pyomgpu_last_error()
void set_last_error(const char* msg) { g_last_error = msg; }
// grid size and the 1-D device metrics (dxt, dxu, dyt, dyu, cost, cosu; index Fortran + 1) of a context
int ctx_grid1d(pyomgpu_ctx* c, int* nx, int* ny, const double** out6, int* cyclic_x, int* cyclic_y) {
  if (!c) return fail(PYOMGPU_EINVAL, "null context");
  *nx = c->nx;
  *ny = c->ny;
  if (cyclic_x) *cyclic_x = c->g.cyclic_x;
  if (cyclic_y) *cyclic_y = c->g.cyclic_y;
  const double* a[6] = {c->dxt, c->dxu, c->dyt, c->dyu, c->cost, c->cosu};
  for (int k = 0; k < 6; k++) out6[k] = a[k];
  return PYOMGPU_OK;
}
}  // namespace pyomgpu

// struct pyomgpu_ctx lives in ctx.h

namespace {

int upload(double** d, const double* h, size_t n) {
  if (int rc = dalloc(d, n)) return rc;
  if (h)
    CK(cudaMemcpy(*d, h, n * sizeof(double), cudaMemcpyHostToDevice));
  else
    CK(cudaMemset(*d, 0, n * sizeof(double)));
  return 0;
}

// Stage a Fortran-layout (nx+4, ny+4) array: device pointers pass through,
// host pointers are copied into `stage`.
int stage_in(pyomgpu_ctx* c, const double* user, double* stage, const double** out, cudaStream_t st) {
  if (is_device_ptr(user)) {
    *out = user;
    return 0;
  }
  CK(cudaMemcpyAsync(stage, user, c->n2 * sizeof(double), cudaMemcpyHostToDevice, st));
  *out = stage;
  return 0;
}

// Waits for a CG launch bracketed by c->e0/e1 and fills info from its result.
int finish_cg(pyomgpu_ctx* c, pyomgpu_solve_info* info, cudaStream_t st) {
  CK(cudaMemcpyAsync(c->h_result, c->d_result, sizeof(CGResult), cudaMemcpyDeviceToHost, st));
  int err = 0;
  CK(cudaMemcpyAsync(c->h_scal, &c->ctl->error, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::memcpy(&err, c->h_scal, sizeof(int));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->e0, c->e1));
  if (info) {
    info->iterations = c->h_result->iterations;
    info->converged = c->h_result->converged;
    info->status = c->h_result->status;
    info->outer_iterations = 1;
    info->estimated_error = c->h_result->est;
    info->rel_residual = -1.0;
    info->device_ms = ms;
    info->kernel_launches = 1;
    if (err) {
      info->status = PYOMGPU_TIMEOUT;
      info->converged = 0;
    }
  }
  if (err) return fail(PYOMGPU_TIMEOUT, "grid barrier wait exceeded %.3f s", c->timeout_s);
  return c->h_result->status;
}

// Estimated iteration time (ns) of the FP64 resident kernel on a w x h piece
// at p points per thread with nb blocks, fitted to the 1440x720 solve timed
// under all 18 cuts that fit at 16 points per thread (8.9-10.2 us, fit within
// ~0.2 us): a constant, the piece's points, the cache lines its exchange
// records occupy (a west or east record on a line of its own, south and north
// ones four to a line), the warps whose threads span two column segments
// (e.g. 39-wide pieces: 11 of 15; 160-wide: none) and the reduction slots.
// f32: the FP32 kernel, whose pieces are counted at their thread capacity
// (threads x points per thread): at 32 points per thread a thread's rows set
// the sweep time, and 1440x720 on 8 x 18 pieces of 180 x 40 (360 threads x
// 32) ran 11.6 us per iteration against 8.5 us on 16-point cuts of the same
// piece size.  With that the same estimate ranks the FP32 cuts as measured
// (five cuts each of 1440x720 and 2048x1024, within ~0.5 us).
double res_iter_ns(int w, int h, int p, int nb, bool f32 = false) {
  const int thr = res_threads(w, h, p);
  int straddle = 0;
  for (int t0 = 0; t0 < thr; t0 += 32)
    if (t0 / w != std::min(t0 + 31, thr - 1) / w) straddle++;
  const double pts = f32 ? (double)thr * p : (double)w * h;
  return 3480.0 + 0.49 * pts + 1.86 * (2.0 * h + 0.5 * w) + 42.0 * straddle + 10.4 * nb;
}

// Cut of an nx x ny grid into npx x npy pieces for the resident kernel: among
// the cuts into at most maxb pieces (pieces at least 2 x 2) whose largest piece
// fits in `cap` bytes of dynamic shared memory and in the worker threads at p
// points per thread (p = 0: the smallest instance that fits), the one with
// the smallest estimated iteration time (res_iter_ns), or with
// least_block_time the smallest iteration time x pieces.  cost: the
// estimate.  False when none fits.
struct ResCut {
  int npx = 0, npy = 0, w = 0, h = 0, p = 0;
  size_t smem = 0;
  double cost = 1e300;
};
bool res_cut(int nx, int ny, int maxb, size_t cap, int p_fixed, bool least_block_time, ResCut& out,
             bool f32 = false) {
  out = ResCut{};
  static constexpr int kP32[] = {16, 32};  // FP32 instances (cg_res32_kernel)
  const int* plist = f32 ? kP32 : kResP;
  const int np = f32 ? 2 : kResNP;
  double best = 1e300;
  for (int npx = 1; npx <= std::min(nx / 2, maxb); npx++)
    for (int npy = 1; npy <= ny / 2 && npx * npy <= maxb; npy++) {
      const int w = (nx + npx - 1) / npx, h = (ny + npy - 1) / npy;
      const size_t bytes = f32 ? res32_smem_bytes(w, h) : res_smem_bytes(w, h);
      if (bytes > cap || w + h > kResWorkers) continue;
      int pp = 0;
      for (int k = 0; k < np && !pp; k++)
        if ((p_fixed == 0 || plist[k] == p_fixed) && res_threads(w, h, plist[k]) <= kResWorkers) pp = plist[k];
      if (!pp) continue;
      const int nb = npx * npy;
      const double cost = res_iter_ns(w, h, pp, nb, f32);
      const double key = least_block_time ? cost * nb : cost;
      if (key < best) {
        best = key;
        out.npx = npx;
        out.npy = npy;
        out.w = w;
        out.h = h;
        out.p = pp;
        out.smem = bytes;
        out.cost = cost;
      }
    }
  return out.npx > 0;
}

// Dynamic shared memory the resident kernels may use on this device: the
// opt-in limit less the largest static shared memory among them (0: none).
size_t res_smem_cap(pyomgpu_ctx* c) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) != cudaSuccess) return 0;
  size_t stat = 0;
  std::vector<const void*> ks{cg_res_multi_kernel_ptr(false), cg_res_multi_kernel_ptr(true), cg_res32_kernel_ptr(16),
                              cg_res32_kernel_ptr(32)};
  for (int k = 0; k < kResNP; k++)
    for (bool single : {false, true}) ks.push_back(cg_res_kernel_ptr(kResP[k], single));
  for (const void* k : ks) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) return 0;
    stat = std::max(stat, fa.sharedSizeBytes);
  }
  return (size_t)optin > stat ? (size_t)optin - stat : 0;
}

// Piece layout of the resident kernel for this grid, planned once (res_cut
// with at most one piece per SM).  Allocates the exchange buffers.  Returns
// PYOMGPU_OK with c->resd.ok telling whether the grid fits, or an error code.
int res_plan(pyomgpu_ctx* c) {
  auto& R = c->resd;
  if (R.planned) return PYOMGPU_OK;
  R.planned = true;
  R.ok = false;
  const size_t cap = res_smem_cap(c);
  if (cap == 0) return PYOMGPU_OK;
  const int maxb = std::min(c->nsm, kResMaxSlots - 1);
  ResCut cut;
  const double best = res_cut(c->nx, c->ny, maxb, cap, 0, false, cut) ? cut.cost : 1e300;
  if (best < 1e300) {
    R.npx = cut.npx;
    R.npy = cut.npy;
    R.wmax = cut.w;
    R.hmax = cut.h;
    R.p = cut.p;
    R.smem = cut.smem;
  }
  if (best == 1e300) return PYOMGPU_OK;
  for (int k = 0; k < kResNP; k++)
    for (bool single : {false, true})
      if (cudaFuncSetAttribute(cg_res_kernel_ptr(kResP[k], single), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)cap) != cudaSuccess)
        return fail(PYOMGPU_ECUDA, "cannot reserve shared memory for the resident kernel");
  for (int k = 0; k < kResNP; k++)
    if (cudaFuncSetAttribute(cg_res_trace_kernel_ptr(kResP[k]), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)cap) != cudaSuccess)
      return fail(PYOMGPU_ECUDA, "cannot reserve shared memory for the resident kernel");
  for (bool single : {false, true}) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_res_kernel_ptr(R.p, single), kResThreads,
                                                      R.smem) != cudaSuccess ||
        per_sm < 1)
      return PYOMGPU_OK;
  }
  const int nb = R.npx * R.npy;
  if (int rc = dalloc(&R.hx, 8 * c->g.size())) return rc;  // two record buffers
  if (int rc = dalloc(&R.slots, (size_t)4 * (nb + 1) * kResSlotWords)) return rc;
  R.ok = true;
  return PYOMGPU_OK;
}

bool use_resident(pyomgpu_ctx* c) {
  if (c->cg_kernel == 1) return false;
  return res_plan(c) == PYOMGPU_OK && c->resd.ok;
}

// The streamfunction solve in the on-chip-resident kernel (cg_res.cu).
int run_cg_res(pyomgpu_ctx* c, const double* forc_dev, double eps, int max_it, double rtol, pyomgpu_solve_info* info,
               cudaStream_t st) {
  auto& R = c->resd;
  const size_t bytes = c->g.size() * sizeof(double);
  const int nb = R.npx * R.npy;
  CK(cudaMemsetAsync(c->ctl, 0, sizeof(SyncCtl), st));
  CK(cudaMemsetAsync(c->res, 0, bytes, st));
  CK(cudaMemsetAsync(R.slots, 0xFF, (size_t)4 * (nb + 1) * kResSlotWords * sizeof(double), st));
  // exchange records all-ones: a word whose tag no solve uses (fresh memory reads as zero, the tag of
  // generation 0, epoch 0, and the untagged single-reduction kernel leaves arbitrary bits)
  CK(cudaMemsetAsync(R.hx, 0xFF, 8 * c->g.size() * sizeof(double), st));
  CGResParams P{};
  P.g = c->g;
  P.op = c->sf.dev();
  P.forc = forc_dev;
  P.sol = c->sol;
  P.res = c->res;
  P.hx = R.hx;
  P.hsize = (long long)c->g.size();
  P.slots = R.slots;
  P.nslot = nb + 1;
  P.npx = R.npx;
  P.npy = R.npy;
  P.wmax = R.wmax;
  P.hmax = R.hmax;
  P.eps = eps;
  P.rtol = rtol;
  P.max_it = max_it;
  P.ctl = c->ctl;
  P.timeout_ns = (unsigned long long)(c->timeout_s * 1e9);
  P.stall_extra = c->stall_next;
  c->stall_next = 0;
  P.tag_gen = R.tag_gen;  // tags of this solve's slots and records differ from the previous solve's
  R.tag_gen = (R.tag_gen + 1u) % 4095u;
  P.out = c->d_result;
  const bool trace = R.trace_nit > 0 && c->cg_kernel != 3;
  P.trace = trace ? R.trace : nullptr;
  P.trace_it0 = R.trace_it0;
  P.trace_nit = trace ? R.trace_nit : 0;
  void* args[] = {&P};
  CK(cudaEventRecord(c->e0, st));
  const bool single = c->cg_kernel == 3;  // automatic: the two-reduction form (the reference's recurrences)
  const void* kern = trace ? cg_res_trace_kernel_ptr(R.p) : cg_res_kernel_ptr(R.p, single);
  CK(cudaLaunchCooperativeKernel(kern, dim3(nb), dim3(kResThreads), args, R.smem, st));
  CK(cudaEventRecord(c->e1, st));
  return finish_cg(c, info, st);
}

// Piece layout of the FP32 resident kernel for this grid (res_cut with FP32
// fields), planned once, with its exchange buffers.  c->resd.ok32 tells
// whether the grid fits.
int res_plan32(pyomgpu_ctx* c) {
  auto& R = c->resd;
  if (R.planned32) return PYOMGPU_OK;
  R.planned32 = true;
  R.ok32 = false;
  const size_t cap = res_smem_cap(c);
  if (cap == 0) return PYOMGPU_OK;
  ResCut cut;
  if (!res_cut(c->nx, c->ny, std::min(c->nsm, kResMaxSlots - 1), cap, 0, false, cut, true)) return PYOMGPU_OK;
  for (int p : {16, 32})
    if (cudaFuncSetAttribute(cg_res32_kernel_ptr(p), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap) !=
        cudaSuccess)
      return fail(PYOMGPU_ECUDA, "cannot reserve shared memory for the FP32 resident kernel");
  const int nb = cut.npx * cut.npy;
  if (int rc = dalloc(&R.hx32, 2 * c->g.size())) return rc;  // two tagged words per position
  if (int rc = dalloc(&R.slots32, (size_t)4 * (nb + 1) * kResSlotWords)) return rc;
  if (int rc = dalloc(&R.res32, c->g.size())) return rc;
  R.npx32 = cut.npx;
  R.npy32 = cut.npy;
  R.wmax32 = cut.w;
  R.hmax32 = cut.h;
  R.p32 = cut.p;
  R.smem32 = cut.smem;
  R.ok32 = true;
  return PYOMGPU_OK;
}

// The FP32 correction solve of the mixed-precision path on the resident
// kernel: A x = b with the FP32 operator copy, b and x padded (x halo valid,
// here zero), to ||res|| <= rtol ||b|| over the unknowns.  Same result
// fields as run_pipe.
int run_cg_res32(pyomgpu_ctx* c, const OpDev<float>& op, const float* b, float* x, double rtol, int max_it,
                 PipeResult* res, float* ms, cudaStream_t st) {
  auto& R = c->resd;
  const int nb = R.npx32 * R.npy32;
  CK(cudaMemsetAsync(c->ctl, 0, sizeof(SyncCtl), st));
  CK(cudaMemsetAsync(R.res32, 0, c->g.size() * sizeof(float), st));
  CK(cudaMemsetAsync(R.slots32, 0xFF, (size_t)4 * (nb + 1) * kResSlotWords * sizeof(double), st));
  CK(cudaMemsetAsync(R.hx32, 0xFF, 2 * c->g.size() * sizeof(double), st));
  CGResParams P{};
  P.g = c->g;
  P.op32 = op;
  P.forc32 = b;
  P.sol32 = x;
  P.res32 = R.res32;
  P.hx = R.hx32;
  P.hsize = (long long)c->g.size();
  P.slots = R.slots32;
  P.nslot = nb + 1;
  P.npx = R.npx32;
  P.npy = R.npy32;
  P.wmax = R.wmax32;
  P.hmax = R.hmax32;
  P.eps = 0.0;
  P.rtol = rtol;
  P.max_it = max_it;
  P.ctl = c->ctl;
  P.timeout_ns = (unsigned long long)(c->timeout_s * 1e9);
  P.out = c->d_result;
  void* args[] = {&P};
  CK(cudaEventRecord(c->e0, st));
  CK(cudaLaunchCooperativeKernel(cg_res32_kernel_ptr(R.p32), dim3(nb), dim3(kResThreads), args, R.smem32, st));
  CK(cudaEventRecord(c->e1, st));
  CK(cudaMemcpyAsync(c->h_result, c->d_result, sizeof(CGResult), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(c->h_scal, &c->ctl->error, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  int err = 0;
  std::memcpy(&err, c->h_scal, sizeof(int));
  if (err) return fail(PYOMGPU_TIMEOUT, "reduction wait exceeded %.3f s", c->timeout_s);
  CK(cudaEventElapsedTime(ms, c->e0, c->e1));
  res->iterations = c->h_result->iterations;
  res->status = c->h_result->status;
  res->rr = res->bb = -1.0;
  return 0;
}

// Runs the persistent CG kernel on c->sol (padded, already packed) with the
// Fortran-layout device forcing.  Fills info (iterations, status, timing).
int run_cg_ref(pyomgpu_ctx* c, bool surf_press, const double* forc_dev, double eps, int max_it, double rtol,
               pyomgpu_solve_info* info, cudaStream_t st) {
  if (!surf_press && use_resident(c)) return run_cg_res(c, forc_dev, eps, max_it, rtol, info, st);
  const OpBuf& op = surf_press ? c->sp : c->sf;
  const size_t bytes = c->g.size() * sizeof(double);
  CK(cudaMemsetAsync(c->ctl, 0, sizeof(SyncCtl), st));
  CK(cudaMemsetAsync(c->res, 0, bytes, st));
  CK(cudaMemsetAsync(c->s0, 0, bytes, st));
  CK(cudaMemsetAsync(c->s1, 0, bytes, st));
  CGRefParams P{};
  P.g = c->g;
  P.op = op.dev();
  const int tx = c->tune.done ? c->tune.tx : kTileX, ty = c->tune.done ? c->tune.ty : kTileY;
  const int bx = tx + 4, by = ty + 2;
  if (encode_tile_map(&P.map_res, c->res, c->g, bx, by) || encode_tile_map(&P.map_W, op.W, c->g, bx, by) ||
      encode_tile_map(&P.map_FX, op.FX, c->g, bx, by) || encode_tile_map(&P.map_FY, op.FY, c->g, bx, by) ||
      encode_tile_map(&P.map_s[0], c->s0, c->g, bx, by) || encode_tile_map(&P.map_s[1], c->s1, c->g, bx, by))
    return fail(PYOMGPU_ECUDA, "cuTensorMapEncodeTiled failed");
  P.tx = tx;
  P.ty = ty;
  P.ntx = (c->nx + tx - 1) / tx;
  P.nty = (c->ny + ty - 1) / ty;
  const int grid = c->tune.done ? c->tune.grid : std::max(1, std::min(c->max_blocks, P.ntx * P.nty));
  P.forc = forc_dev;
  P.sol = c->sol;
  P.res = c->res;
  P.s[0] = c->s0;
  P.s[1] = c->s1;
  P.As = c->As;
  P.eps = eps;
  P.max_it = max_it;
  P.rtol = rtol;
  P.ctl = c->ctl;
  P.slots = c->slots;
  P.timeout_ns = (unsigned long long)(c->timeout_s * 1e9);
  P.stall_extra = c->stall_next;
  c->stall_next = 0;
  P.out = c->d_result;
  void* args[] = {&P};
  CK(cudaEventRecord(c->e0, st));
  CK(cudaLaunchCooperativeKernel(cg_ref_kernel_ptr(surf_press), dim3(grid), dim3(kCGThreads), args,
                                 cg_smem_bytes(tx, ty), st));
  CK(cudaEventRecord(c->e1, st));
  return finish_cg(c, info, st);
}

}  // namespace

int run_pcg_from_sol(pyomgpu_ctx* c, const double* forc_dev, int max_it, double rtol, pyomgpu_solve_info* info,
                     cudaStream_t st) {
  return run_cg_ref(c, false, forc_dev, 0.0, max_it, rtol, info, st);
}

namespace {

template <typename T>
int fast_alloc(pyomgpu_ctx* c, T** p, size_t n) {
  if (int rc = dalloc(p, n)) return rc;
  c->fast.owned.push_back(*p);
  return 0;
}

// Buffers of the single-barrier PCG; FP32 operator and vectors when f32.
int fast_setup(pyomgpu_ctx* c, bool f32, cudaStream_t st) {
  auto& F = c->fast;
  const size_t P = c->g.size();
  int rc;
  if (!F.ready) {
    int o1 = 0, o2 = 0;
    for (bool f : {false, true})
      if (cudaFuncSetAttribute(cg_pipe_kernel_ptr(f), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)pipe_smem_bytes(f)) != cudaSuccess)
        return fail(PYOMGPU_ECUDA, "cannot reserve shared memory for the pipelined kernel");
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, cg_pipe_kernel_ptr(false), kPipeThreads,
                                                      pipe_smem_bytes(false)) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, cg_pipe_kernel_ptr(true), kPipeThreads,
                                                      pipe_smem_bytes(true)) ||
        o1 < 1 || o2 < 1)
      return fail(PYOMGPU_ECUDA, "occupancy query failed");
    F.max_blocks = std::min(o1, o2) * c->nsm;
    if ((rc = fast_alloc(c, &F.b, P)) || (rc = fast_alloc(c, &F.r[0], P)) || (rc = fast_alloc(c, &F.r[1], P)) ||
        (rc = fast_alloc(c, &F.q[0], P)) || (rc = fast_alloc(c, &F.q[1], P)) || (rc = fast_alloc(c, &F.w[0], P)) ||
        (rc = fast_alloc(c, &F.w[1], P)) || (rc = fast_alloc(c, &F.p, P)) ||
        (rc = fast_alloc(c, &F.slots, (size_t)2 * F.max_blocks * 8)) || (rc = fast_alloc(c, &F.d_res, 1)))
      return rc;
    if (cudaMallocHost((void**)&F.h_res, sizeof(PipeResult)) != cudaSuccess)
      return fail(PYOMGPU_ENOMEM, "cudaMallocHost");
    F.ready = true;
  }
  if (f32 && !F.f32_ready) {
    const size_t X = c->nx + 4, Y = c->ny + 4;
    if ((rc = fast_alloc(c, &F.FX, P)) || (rc = fast_alloc(c, &F.FY, P)) || (rc = fast_alloc(c, &F.W, P)) ||
        (rc = fast_alloc(c, &F.ax, X)) || (rc = fast_alloc(c, &F.bx, Y)) || (rc = fast_alloc(c, &F.by, Y)) ||
        (rc = fast_alloc(c, &F.b32, P)) || (rc = fast_alloc(c, &F.x32, P)) || (rc = fast_alloc(c, &F.p32, P)) ||
        (rc = fast_alloc(c, &F.r32[0], P)) || (rc = fast_alloc(c, &F.r32[1], P)) ||
        (rc = fast_alloc(c, &F.q32[0], P)) || (rc = fast_alloc(c, &F.q32[1], P)) ||
        (rc = fast_alloc(c, &F.w32[0], P)) || (rc = fast_alloc(c, &F.w32[1], P)))
      return rc;
    F.f32_ready = true;
  }
  if (f32 && F.op32_stale) {  // FP32 copy of the streamfunction operator (Z included)
    F.op32_stale = false;
    launch_to_f32(c->sf.FX, F.FX, P, st);
    launch_to_f32(c->sf.FY, F.FY, P, st);
    launch_to_f32(c->sf.W, F.W, P, st);
    launch_to_f32(c->sf.ax, F.ax, (size_t)c->nx + 4, st);
    launch_to_f32(c->sf.bx, F.bx, (size_t)c->ny + 4, st);
    launch_to_f32(c->sf.by, F.by, (size_t)c->ny + 4, st);
    F.op32 = OpDev<float>{F.FX, F.FY, F.ax, F.bx, F.by, F.W, 0.f};
  }
  return 0;
}

// One launch of the pipelined PCG on (b, x) with the given buffers (x's halo valid).
template <typename T>
int run_pipe(pyomgpu_ctx* c, const OpDev<T>& op, const T* b, T* x, T* const r[2], T* const A[2], T* const s[2],
             double rtol, int max_it, PipeResult* res, float* ms, cudaStream_t st) {
  auto& F = c->fast;
  const size_t bytes = c->g.size() * sizeof(T);
  CK(cudaMemsetAsync(c->ctl, 0, sizeof(SyncCtl), st));
  for (T* a : {r[0], r[1], A[0], A[1], s[0], s[1]}) CK(cudaMemsetAsync(a, 0, bytes, st));
  PipeParams<T> P{};
  P.g = c->g;
  P.op = op;
  P.b = b;
  P.x = x;
  for (int k = 0; k < 2; k++) {
    P.r[k] = r[k];
    P.A[k] = A[k];
    P.s[k] = s[k];
  }
  if (pipe_encode_all(P)) return fail(PYOMGPU_ECUDA, "cuTensorMapEncodeTiled failed");
  P.rtol = rtol;
  P.max_it = max_it;
  P.ntx = (c->nx + kTileX - 1) / kTileX;
  P.nty = (c->ny + kTileY - 1) / kTileY;
  const int grid = std::max(1, std::min(F.max_blocks, P.ntx * P.nty));
  P.ctl = c->ctl;
  P.slots = F.slots;
  P.timeout_ns = (unsigned long long)(c->timeout_s * 1e9);
  P.out = F.d_res;
  void* args[] = {&P};
  CK(cudaEventRecord(c->e0, st));
  CK(cudaLaunchCooperativeKernel(cg_pipe_kernel_ptr(sizeof(T) == 4), dim3(grid), dim3(kPipeThreads), args,
                                 pipe_smem_bytes(sizeof(T) == 4), st));
  CK(cudaEventRecord(c->e1, st));
  CK(cudaMemcpyAsync(F.h_res, F.d_res, sizeof(PipeResult), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(c->h_scal, &c->ctl->error, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  int err = 0;
  std::memcpy(&err, c->h_scal, sizeof(int));
  if (err) return fail(PYOMGPU_TIMEOUT, "grid barrier wait exceeded %.3f s", c->timeout_s);
  CK(cudaEventElapsedTime(ms, c->e0, c->e1));
  *res = *F.h_res;
  return 0;
}

// One solve of a batch: its grid/operator context and its device Fortran-layout
// forcing (NULL = zero) and solution (in/out).
struct BatchSpec {
  pyomgpu_ctx* c;
  const double* forc;
  double* sol;
};

inline size_t align32(size_t n) { return (n + 31) / 32 * 32; }

// Work-pool words of one solve of pyomgpu_congrad_streamfunction_batch, enough
// for either engine: the work-queue kernel's padded sol, res, s0, s1, As, or
// the resident groups' padded sol, res, 4 record words per position and the
// reduction slots.  The staged host inputs follow the work space of all solves.
inline size_t batch_job_words(size_t padded) {
  return std::max(5 * align32(padded), 6 * align32(padded) + align32((size_t)4 * kResMaxSlots * kResSlotWords));
}

// Grows the owner's batch workspace for `count` solves needing `pool` doubles and `tasks` tiles.
int batch_reserve(pyomgpu_ctx* o, int count, size_t pool, size_t tasks) {
  auto& B = o->batch;
  if (!B.sync) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_batch_kernel_ptr(), kBatchThreads, 0) !=
            cudaSuccess ||
        per_sm < 1)
      return fail(PYOMGPU_ECUDA, "occupancy query of the batch kernel failed");
    B.max_blocks = per_sm * o->nsm;
    int l2 = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, o->device) != cudaSuccess) l2 = 0;
    B.l2_bytes = (size_t)std::max(l2, 0);
    if (int rc = dalloc(&B.sync, 8)) return rc;
  }
  if (pool > B.cap) {
    if (B.pool) cudaFree(B.pool);
    B.pool = nullptr;
    B.cap = 0;
    if (int rc = dalloc(&B.pool, pool)) return rc;
    B.cap = pool;
  }
  if (count > B.cap_probs) {
    if (B.d_probs) cudaFree(B.d_probs);
    if (B.h_probs) cudaFreeHost(B.h_probs);
    if (B.d_state) cudaFree(B.d_state);
    if (B.h_state) cudaFreeHost(B.h_state);
    if (B.d_rr) cudaFree(B.d_rr);
    if (B.h_rr) cudaFreeHost(B.h_rr);
    if (B.d_act) cudaFree(B.d_act);
    if (B.h_act) cudaFreeHost(B.h_act);
    B.d_probs = nullptr;
    B.h_probs = nullptr;
    B.d_state = nullptr;
    B.h_state = nullptr;
    B.d_rr = B.h_rr = nullptr;
    B.d_act = B.h_act = nullptr;
    B.cap_probs = 0;
    if (int rc = dalloc(&B.d_probs, (size_t)count)) return rc;
    if (int rc = dalloc(&B.d_state, (size_t)count)) return rc;
    if (int rc = dalloc(&B.d_rr, (size_t)count * 2)) return rc;
    if (int rc = dalloc(&B.d_act, (size_t)3 * count + 2)) return rc;
    if (cudaMallocHost((void**)&B.h_probs, sizeof(BatchProblem) * count) != cudaSuccess ||
        cudaMallocHost((void**)&B.h_state, sizeof(BatchState) * count) != cudaSuccess ||
        cudaMallocHost((void**)&B.h_rr, sizeof(double) * 2 * count) != cudaSuccess ||
        cudaMallocHost((void**)&B.h_act, sizeof(int) * (2 * count + 2)) != cudaSuccess)
      return fail(PYOMGPU_ENOMEM, "cudaMallocHost");
    B.cap_probs = count;
  }
  if (tasks > B.cap_tasks) {
    if (B.part) cudaFree(B.part);
    B.part = nullptr;
    B.cap_tasks = 0;
    if (int rc = dalloc(&B.part, tasks * 4)) return rc;
    B.cap_tasks = tasks;
  }
  return 0;
}

// Runs the solves of `v` in one launch of the work-queue kernel with the
// workspace of `o`.  infos (v.size() entries) get each solve's result; with
// want_res the FP64 true relative residual of each solution as well.
int run_batch(pyomgpu_ctx* o, const std::vector<BatchSpec>& v, double eps, int max_it, double rtol, bool want_res,
              pyomgpu_solve_info* infos, float* ms_out, cudaStream_t st, int weighted = 0) {
  const int count = (int)v.size();
  if (count > kBatchActMax) {  // one launch per kBatchActMax solves
    int worst = PYOMGPU_OK;
    float total = 0.f;
    for (int k0 = 0; k0 < count; k0 += kBatchActMax) {
      const std::vector<BatchSpec> sub(v.begin() + k0, v.begin() + std::min(count, k0 + kBatchActMax));
      float ms = 0.f;
      const int rc = run_batch(o, sub, eps, max_it, rtol, want_res, infos ? infos + k0 : nullptr, &ms, st, weighted);
      if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
      worst = std::max(worst, rc);
      total += ms;
    }
    if (ms_out) *ms_out = total;
    return worst;
  }
  size_t pool = 0, tasks = 0;
  for (const BatchSpec& b : v) {
    pool += 5 * align32(b.c->g.size());
    tasks += (size_t)((b.c->nx + kTileX - 1) / kTileX) * ((b.c->ny + kTileY - 1) / kTileY);
  }
  if (tasks > (size_t)0x7fffffff) return fail(PYOMGPU_EINVAL, "batch too large");
  if (int rc = batch_reserve(o, count, pool, tasks)) return rc;
  auto& B = o->batch;
  CK(cudaMemsetAsync(B.pool, 0, pool * sizeof(double), st));
  CK(cudaMemsetAsync(B.sync, 0, 8 * sizeof(unsigned long long), st));
  // all problems in one launch, largest first: every sweep and barrier serves every
  // problem still running, so the barrier latency is shared by all of them (solving
  // L2-sized groups one after another measured slower: each group then pays the
  // latency-bound iterations of its slowest problem on its own)
  std::vector<int> order((size_t)count);
  for (int k = 0; k < count; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return v[a].c->g.size() > v[b].c->g.size(); });
  // the initial active list: every problem, tiles in order
  int* h_actn = B.h_act;
  int* h_actprob = B.h_act + 1;
  int* h_actoff = B.h_act + 1 + count;
  h_actn[0] = count;
  h_actoff[0] = 0;
  double* cur = B.pool;
  int tile0 = 0;
  for (int pos = 0; pos < count; ++pos) {
    const int k = order[pos];
    const BatchSpec& b = v[k];
    const size_t P = align32(b.c->g.size());
    BatchProblem pr{};
    pr.g = b.c->g;
    pr.op = b.c->sf.dev();
    pr.forc = b.forc ? b.forc : b.c->zeros;
    pr.sol = cur;
    pr.res = cur + P;
    pr.s[0] = cur + 2 * P;
    pr.s[1] = cur + 3 * P;
    pr.As = cur + 4 * P;
    cur += 5 * P;
    pr.eps = eps;
    pr.rtol = rtol;
    pr.max_it = max_it;
    pr.weighted = weighted;
    pr.ntx = (b.c->nx + kTileX - 1) / kTileX;
    pr.nty = (b.c->ny + kTileY - 1) / kTileY;
    pr.tile0 = tile0;
    tile0 += pr.ntx * pr.nty;
    B.h_probs[pos] = pr;
    h_actprob[pos] = pos;
    h_actoff[pos + 1] = tile0;
    launch_pack(b.c->g, b.sol, pr.sol, true, st);  // setcyclic_xy(sol), solve_streamfct.f90:191-192
  }
  CK(cudaMemcpyAsync(B.d_probs, B.h_probs, sizeof(BatchProblem) * count, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(B.d_act, B.h_act, sizeof(int) * (2 * count + 2), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(B.d_act + 2 * count + 2, 0, sizeof(int) * count, st));  // per-problem tile counters
  CK(cudaMemsetAsync(B.d_state, 0, sizeof(BatchState) * count, st));
  BatchParams P{};
  P.probs = B.d_probs;
  P.state = B.d_state;
  P.nprob = count;
  P.ntasks = tile0;
  P.part = B.part;
  P.act_n = B.d_act;
  P.act_prob = B.d_act + 1;
  P.act_off = B.d_act + 1 + count;
  P.done = B.d_act + 2 * count + 2;
  P.ctl = reinterpret_cast<SyncCtl*>(B.sync);
  P.gen = B.sync + 2;
  P.timeout_ns = (unsigned long long)(o->timeout_s * 1e9);
  P.stall_extra = o->stall_next;
  o->stall_next = 0;
  const int grid = std::max(1, std::min(B.max_blocks, tile0));
  CK(cudaEventRecord(o->e0, st));
  CK(launch_cg_batch(P, grid, st));
  CK(cudaEventRecord(o->e1, st));
  CK(cudaMemcpyAsync(B.h_state, B.d_state, sizeof(BatchState) * count, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(o->h_scal, &P.ctl->error, sizeof(int), cudaMemcpyDeviceToHost, st));
  for (int pos = 0; pos < count; ++pos) {
    const int k = order[pos];
    const BatchProblem& pr = B.h_probs[pos];
    if (want_res) {
      launch_fill_cyclic(pr.g, pr.sol, st);
      launch_residual(pr.g, pr.op, pr.forc, pr.sol, v[k].c->part, 1024, B.d_rr + 2 * k, st);
    }
    launch_unpack(pr.g, pr.sol, v[k].sol, false, false, false, st);
  }
  if (want_res) CK(cudaMemcpyAsync(B.h_rr, B.d_rr, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  int err = 0;
  std::memcpy(&err, o->h_scal, sizeof(int));
  if (err) return fail(PYOMGPU_TIMEOUT, "grid barrier wait exceeded %.3f s", o->timeout_s);
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, o->e0, o->e1));
  if (ms_out) *ms_out = ms;
  int worst = PYOMGPU_OK;
  for (int pos = 0; pos < count; ++pos) {
    const int k = order[pos];
    const BatchState& S = B.h_state[pos];
    worst = std::max(worst, S.status);
    if (!infos) continue;
    pyomgpu_solve_info& I = infos[k];
    I.iterations = S.n;
    I.converged = S.converged;
    I.status = S.status;
    I.outer_iterations = 1;
    I.estimated_error = S.est;
    I.device_ms = ms;
    I.kernel_launches = 1;
    if (want_res) {
      const double rr = B.h_rr[2 * k], bb = B.h_rr[2 * k + 1];
      I.rel_residual = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
    } else {
      I.rel_residual = -1.0;
    }
  }
  return worst;
}

// Index words of a multi-solve launch on at most kResMaxSlots blocks: the
// per-block list offsets (kResMaxSlots + 1), the error flag, the per-job join
// counters, then the (job, piece) list entries (at most one per block per job).
inline size_t rmulti_idx_words(int count) {
  return (size_t)kResMaxSlots + 2 + (size_t)count + 2 * (size_t)kResMaxSlots * (size_t)count;
}

// Grows the owner's table for `count` resident jobs.
int rmulti_reserve(pyomgpu_ctx* o, int count) {
  auto& R = o->rmulti;
  if (count <= R.cap) return 0;
  for (void* p : {(void*)R.d_jobs, (void*)R.d_idx, (void*)R.d_out, (void*)R.d_ctl, (void*)R.d_times})
    if (p) cudaFree(p);
  for (void* p : {(void*)R.h_jobs, (void*)R.h_idx, (void*)R.h_out, (void*)R.h_ctl, (void*)R.h_times})
    if (p) cudaFreeHost(p);
  R.d_jobs = nullptr;
  R.h_jobs = nullptr;
  R.d_idx = R.h_idx = nullptr;
  R.d_out = R.h_out = nullptr;
  R.d_ctl = R.h_ctl = nullptr;
  R.d_times = R.h_times = nullptr;
  R.cap = 0;
  if (int rc = dalloc(&R.d_jobs, (size_t)count)) return rc;
  if (int rc = dalloc(&R.d_idx, rmulti_idx_words(count))) return rc;
  if (int rc = dalloc(&R.d_out, (size_t)count)) return rc;
  if (int rc = dalloc(&R.d_ctl, (size_t)count)) return rc;
  if (int rc = dalloc(&R.d_times, (size_t)2 * count)) return rc;
  if (cudaMallocHost((void**)&R.h_jobs, sizeof(CGResParams) * count) != cudaSuccess ||
      cudaMallocHost((void**)&R.h_idx, sizeof(int) * rmulti_idx_words(count)) != cudaSuccess ||
      cudaMallocHost((void**)&R.h_out, sizeof(CGResult) * count) != cudaSuccess ||
      cudaMallocHost((void**)&R.h_ctl, sizeof(SyncCtl) * count) != cudaSuccess ||
      cudaMallocHost((void**)&R.h_times, sizeof(unsigned long long) * 2 * count) != cudaSuccess)
    return fail(PYOMGPU_ENOMEM, "cudaMallocHost");
  R.cap = count;
  return 0;
}

// List scheduling of rigid gangs on nsm blocks: job k needs nb[k] blocks for
// est[k] (any unit).  In a given order each job takes the nb[k] blocks that
// become free earliest (ties: lower block index) and starts when the last of
// them is free.  The order: init (a permutation) or largest gang first, then
// longest; then `tries` seeded local-search steps (a few swaps of nearby jobs,
// kept when the makespan drops).  rank orders the jobs by planned start (ties:
// the final order); a block serving several jobs runs them by rank, one total
// order for all blocks, so gangs cannot wait on one another in a cycle.
struct GangPlan {
  std::vector<int> order, rank;
  std::vector<double> start;
  std::vector<std::vector<int>> gang;  // blocks of each job, ascending (piece q = gang[k][q])
  double makespan = 0.0;
};
void plan_gangs(int nsm, const std::vector<int>& nb, const std::vector<double>& est, const std::vector<int>* init,
                int tries, GangPlan& out) {
  const int count = (int)nb.size();
  // the blocks as (free time, index), kept sorted: a job takes the first nb[k]
  // (the earliest free, lower index first on ties), which all become free at
  // t + est[k] and are merged back into place -- O(nsm) per job, no sort
  std::vector<std::pair<double, int>> fr((size_t)nsm), taken, merged((size_t)nsm);
  out.start.assign((size_t)count, 0.0);
  out.gang.assign((size_t)count, {});
  auto place = [&](const std::vector<int>& ord, bool record) {
    for (int b = 0; b < nsm; ++b) fr[b] = {0.0, b};
    double span = 0.0;
    for (int k : ord) {
      const int n = nb[k];
      const double t = fr[n - 1].first;
      const double done = t + est[k];
      span = std::max(span, done);
      taken.assign(fr.begin(), fr.begin() + n);
      if (record) {
        out.start[k] = t;
        out.gang[k].resize((size_t)n);
        for (int q = 0; q < n; ++q) out.gang[k][q] = taken[q].second;
        std::sort(out.gang[k].begin(), out.gang[k].end());
      }
      for (auto& e : taken) e.first = done;
      std::sort(taken.begin(), taken.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
        return a.second < b.second;  // equal times: by index
      });
      std::merge(fr.begin() + n, fr.end(), taken.begin(), taken.end(), merged.begin());
      fr.swap(merged);
    }
    return span;
  };
  std::vector<int>& order = out.order;
  order.resize((size_t)count);
  if (init) {
    order = *init;
  } else {
    for (int k = 0; k < count; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return nb[a] != nb[b] ? nb[a] > nb[b] : est[a] > est[b]; });
  }
  if (count > 2) {
    double best = place(order, false);
    uint64_t rng = 0x9E3779B97F4A7C15ull;
    auto next = [&rng]() {
      rng ^= rng << 13;
      rng ^= rng >> 7;
      rng ^= rng << 17;
      return rng;
    };
    std::vector<int> cand;
    for (int it = 0; it < tries; ++it) {
      cand = order;
      for (int q = 0; q < 8; ++q) {
        const int i = (int)(next() % (uint64_t)(count - 1));
        const int j = std::min(count - 1, i + 1 + (int)(next() % 5));
        std::swap(cand[i], cand[j]);
      }
      const double span = place(cand, false);
      if (span < best) {
        best = span;
        order.swap(cand);
      }
    }
  }
  out.makespan = place(order, true);
  out.rank.assign((size_t)count, 0);
  std::vector<int> by_start = order;
  std::stable_sort(by_start.begin(), by_start.end(), [&](int a, int b) { return out.start[a] < out.start[b]; });
  for (int r = 0; r < count; ++r) out.rank[by_start[r]] = r;
}

// The solves of `v` on the resident kernel, several at once, in one launch of
// cg_res_multi_kernel on all SMs.  Every solve takes its densest cut (res_cut
// with the least estimated block-time per iteration at 16 points per thread)
// and is placed by list scheduling on the host, largest gangs
// first, then longest, improved by a seeded local search over the order: on
// the pieces' count of blocks that become free earliest under the estimated
// durations (the grid's device time in the
// previous resident batch, measured with %globaltimer around its solve; else
// ~2 x the square root of the point count iterations times the cut's
// iteration estimate); each block runs its
// entries in order of planned start.
// *used = false (nothing run) when a grid does not fit on chip or the
// resident kernel is unavailable; the caller then runs the work-queue kernel.
int run_res_multi(pyomgpu_ctx* o, const std::vector<BatchSpec>& v, double eps, int max_it, double rtol,
                  bool want_res, pyomgpu_solve_info* infos, float* ms_out, cudaStream_t st, bool* used,
                  int weighted = 0) {
  *used = false;
  const int count = (int)v.size();
  auto& R = o->rmulti;
  if (R.smem_cap == 0) {
    const size_t cap = res_smem_cap(o);
    if (cap == 0) return PYOMGPU_OK;
    for (bool w : {false, true})
      if (cudaFuncSetAttribute(cg_res_multi_kernel_ptr(w), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap) !=
          cudaSuccess)
        return PYOMGPU_OK;
    R.smem_cap = cap;
  }
  const int nsm = std::min(o->nsm, kResMaxSlots - 1);
  std::vector<ResCut> cuts((size_t)count);
  std::vector<double> est((size_t)count);
  int need = 0;
  for (int k = 0; k < count; ++k) {
    const pyomgpu_ctx* c = v[k].c;
    if (!res_cut(c->nx, c->ny, nsm, R.smem_cap, 16, true, cuts[k])) return PYOMGPU_OK;
    need += cuts[k].npx * cuts[k].npy;
  }
  // fewer pieces in all than SMs: every solve gets its share of the SMs (in
  // proportion to its densest cut) and the fastest cut within it, all at once
  if (need < nsm) {
    for (int k = 0; k < count; ++k) {
      const pyomgpu_ctx* c = v[k].c;
      const int share = std::max(cuts[k].npx * cuts[k].npy, (nsm * cuts[k].npx * cuts[k].npy) / need);
      ResCut cut;
      if (res_cut(c->nx, c->ny, share, R.smem_cap, 16, false, cut)) cuts[k] = cut;
    }
  } else {
    // a solve beside whose densest cut no other solve of the batch fits takes the
    // fastest cut over all SMs (the rest would idle while it runs)
    std::vector<int> dense((size_t)count);
    for (int k = 0; k < count; ++k) dense[k] = cuts[k].npx * cuts[k].npy;
    for (int k = 0; k < count; ++k) {
      int others = nsm + 1;  // the smallest densest cut among the other solves
      for (int q = 0; q < count; ++q)
        if (q != k) others = std::min(others, dense[q]);
      if (others > nsm - dense[k]) {
        ResCut cut;
        if (res_cut(v[k].c->nx, v[k].c->ny, nsm, R.smem_cap, 16, false, cut)) cuts[k] = cut;
      }
    }
  }
  // estimated duration (ns): this grid's device time in the previous resident batch at the
  // same occurrence, else ~2 sqrt(points) iterations x the cut's iteration estimate
  std::vector<int> occ((size_t)count, 0);
  for (int k = 0; k < count; ++k)
    for (int q = 0; q < k; ++q) occ[k] += v[q].c == v[k].c;
  for (int k = 0; k < count; ++k) {
    const pyomgpu_ctx* c = v[k].c;
    est[k] = occ[k] < (int)c->batch_ns.size() && c->batch_ns[occ[k]] > 0.0
                 ? c->batch_ns[occ[k]]
                 : 2.0 * std::sqrt((double)c->nx * c->ny) * cuts[k].cost;
  }
  // workspace per solve (batch_job_words): padded sol and res, 4 record words per
  // position, the slots; the caller has reserved it before staging its inputs
  // behind it, so the pool is never reallocated here
  size_t pool = 0;
  for (int k = 0; k < count; ++k) pool += batch_job_words(v[k].c->g.size());
  if (pool > o->batch.cap) return fail(PYOMGPU_EINVAL, "resident batch: work pool not reserved");
  if (int rc = batch_reserve(o, count, pool, 1)) return rc;
  if (int rc = rmulti_reserve(o, count)) return rc;
  *used = true;
  auto& B = o->batch;
  CK(cudaMemsetAsync(R.d_ctl, 0, sizeof(SyncCtl) * count, st));  // every solve's error flag
  // every solve's slice of the pool (call order), zeroed residual, all-ones records and
  // slots (no tag of the solve, generation 0), packed first guess: on the stream while the
  // host plans the schedule
  std::vector<double*> slice((size_t)count);
  {
    double* cur = B.pool;
    for (int k = 0; k < count; ++k) {
      const pyomgpu_ctx* c = v[k].c;
      const size_t P = align32(c->g.size());
      slice[k] = cur;
      CK(cudaMemsetAsync(cur + P, 0, P * sizeof(double), st));
      CK(cudaMemsetAsync(cur + 2 * P, 0xFF, (4 * P + (size_t)4 * (nsm + 1) * kResSlotWords) * sizeof(double), st));
      launch_pack(c->g, v[k].sol, cur, true, st);  // setcyclic_xy(sol), solve_streamfct.f90:191-192
      cur += batch_job_words(c->g.size());
    }
  }
  // order: the owner's previous order when the batch has the same solves (the
  // estimates change a little from call to call: fewer tries), else largest first
  std::vector<int> nbk((size_t)count);
  for (int k = 0; k < count; ++k) nbk[k] = cuts[k].npx * cuts[k].npy;
  bool again = (int)o->sched_key.size() == count && (int)o->sched_order.size() == count;
  for (int k = 0; again && k < count; ++k) again = o->sched_key[k] == v[k].c;
  if (again) {
    std::vector<char> seen((size_t)count, 0);
    for (int k : o->sched_order) {
      again = again && k >= 0 && k < count && !seen[k];
      if (!again) break;
      seen[k] = 1;
    }
  }
  GangPlan plan;
  plan_gangs(nsm, nbk, est, again ? &o->sched_order : nullptr,
             again ? std::max(20, std::min(150, 15000 / count)) : std::max(20, std::min(400, 40000 / count)), plan);
  o->sched_key.resize((size_t)count);
  for (int k = 0; k < count; ++k) o->sched_key[k] = v[k].c;
  o->sched_order = plan.order;
  const std::vector<int>& rank = plan.rank;
  const std::vector<std::vector<int>>& gang = plan.gang;
  std::vector<std::vector<std::pair<int, int>>> lists((size_t)nsm);  // (rank, piece) per block
  for (int k = 0; k < count; ++k)
    for (int q = 0; q < (int)gang[k].size(); ++q) lists[gang[k][q]].push_back({rank[k], q});
  int* h_off = R.h_idx;
  int* h_err = R.h_idx + kResMaxSlots + 1;
  int* h_join = h_err + 1;
  int2* h_list = reinterpret_cast<int2*>(h_join + count + (count & 1));  // 8-byte aligned
  (void)h_err;
  std::vector<int> job_of_rank((size_t)count);
  for (int k = 0; k < count; ++k) job_of_rank[rank[k]] = k;
  int nent = 0;
  for (int b = 0; b < nsm; ++b) {
    std::sort(lists[b].begin(), lists[b].end());
    h_off[b] = nent;
    for (const auto& e : lists[b]) h_list[nent++] = make_int2(e.first, e.second);
  }
  h_off[nsm] = nent;
  // the job table in rank order (list entries name ranks)
  size_t smem = 0;
  for (int r = 0; r < count; ++r) {
    const int k = job_of_rank[r];
    const pyomgpu_ctx* c = v[k].c;
    const ResCut& cut = cuts[k];
    const size_t P = align32(c->g.size());
    double* cur = slice[k];
    CGResParams& J = R.h_jobs[r];
    J = CGResParams{};
    J.g = c->g;
    J.op = c->sf.dev();
    J.forc = v[k].forc ? v[k].forc : c->zeros;
    J.sol = cur;
    J.res = cur + P;
    J.hx = cur + 2 * P;
    J.hsize = (long long)c->g.size();
    J.slots = cur + 6 * P;
    J.nslot = cut.npx * cut.npy + 1;
    J.npx = cut.npx;
    J.npy = cut.npy;
    J.wmax = cut.w;
    J.hmax = cut.h;
    J.eps = eps;
    J.rtol = rtol;
    J.max_it = max_it;
    J.ctl = R.d_ctl + k;
    J.timeout_ns = (unsigned long long)(o->timeout_s * 1e9);
    J.stall_extra = o->stall_next;  // test hook: every first reduction awaits a slot nobody writes
    J.weighted = weighted;
    J.out = R.d_out + k;
    smem = std::max(smem, cut.smem);
  }
  o->stall_next = 0;
  const size_t list_words = (size_t)(reinterpret_cast<int*>(h_list + nent) - R.h_idx);
  CK(cudaMemcpyAsync(R.d_jobs, R.h_jobs, sizeof(CGResParams) * count, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(R.d_idx + kResMaxSlots + 1, 0, sizeof(int) * (count + 1), st));  // error flag, join counters
  // offsets, then (after the zeroed error flag and join counters) the entries
  CK(cudaMemcpyAsync(R.d_idx, R.h_idx, sizeof(int) * (kResMaxSlots + 1), cudaMemcpyHostToDevice, st));
  const size_t lst0 = (size_t)(reinterpret_cast<int*>(h_list) - R.h_idx);
  CK(cudaMemcpyAsync(R.d_idx + lst0, h_list, sizeof(int) * (list_words - lst0), cudaMemcpyHostToDevice, st));
  int* d_err = R.d_idx + kResMaxSlots + 1;
  ResMultiParams M{};
  M.jobs = R.d_jobs;
  M.list_off = R.d_idx;
  M.list = reinterpret_cast<const int2*>(R.d_idx + lst0);
  M.join = d_err + 1;
  M.times = R.d_times;
  M.error = d_err;
  // a block may wait for its gang while other pieces finish their previous solves
  M.gang_timeout_ns = (unsigned long long)(std::max(120.0, 64.0 * o->timeout_s) * 1e9);
  void* args[] = {&M};
  CK(cudaEventRecord(o->e0, st));
  CK(cudaLaunchCooperativeKernel(cg_res_multi_kernel_ptr(weighted != 0), dim3(nsm), dim3(kResThreads), args, smem,
                                 st));
  CK(cudaEventRecord(o->e1, st));
  CK(cudaMemcpyAsync(R.h_out, R.d_out, sizeof(CGResult) * count, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(R.h_ctl, R.d_ctl, sizeof(SyncCtl) * count, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(R.h_idx, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(R.h_times, R.d_times, sizeof(unsigned long long) * 2 * count, cudaMemcpyDeviceToHost, st));
  for (int r = 0; r < count; ++r) {
    const int k = job_of_rank[r];
    const CGResParams& J = R.h_jobs[r];
    if (want_res) {
      launch_fill_cyclic(J.g, J.sol, st);
      launch_residual(J.g, J.op, J.forc, J.sol, v[k].c->part, 1024, B.d_rr + 2 * k, st);
    }
    launch_unpack(J.g, J.sol, v[k].sol, false, false, false, st);
  }
  if (want_res) CK(cudaMemcpyAsync(B.h_rr, B.d_rr, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  if (R.h_idx[0]) return fail(PYOMGPU_TIMEOUT, "resident batch: a gang did not assemble in time");
  for (int k = 0; k < count; ++k)
    if (R.h_ctl[k].error) return fail(PYOMGPU_TIMEOUT, "reduction wait exceeded %.3f s", o->timeout_s);
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, o->e0, o->e1));
  if (ms_out) *ms_out = ms;
  {
    unsigned long long t_min = ~0ull;
    for (int k = 0; k < count; ++k) t_min = std::min(t_min, R.h_times[2 * rank[k]]);
    o->sched_start.assign((size_t)count, 0.0);
    o->sched_end.assign((size_t)count, 0.0);
    o->sched_blocks.assign((size_t)count, 0);
    for (int k = 0; k < count; ++k) {
      o->sched_start[k] = (double)(R.h_times[2 * rank[k]] - t_min) * 1e-6;
      o->sched_end[k] = (double)(R.h_times[2 * rank[k] + 1] - t_min) * 1e-6;
      o->sched_blocks[k] = cuts[k].npx * cuts[k].npy;
    }
  }
  int worst = PYOMGPU_OK;
  for (int k = 0; k < count; ++k) {
    const CGResult& r = R.h_out[k];
    worst = std::max(worst, r.status);
    auto& hist = v[k].c->batch_ns;
    if ((int)hist.size() <= occ[k]) hist.resize((size_t)occ[k] + 1, 0.0);
    const unsigned long long t0 = R.h_times[2 * rank[k]], t1 = R.h_times[2 * rank[k] + 1];
    hist[occ[k]] = t1 > t0 ? (double)(t1 - t0) : 0.0;
    if (!infos) continue;
    pyomgpu_solve_info& I = infos[k];
    I.iterations = r.iterations;
    I.converged = r.converged;
    I.status = r.status;
    I.outer_iterations = 1;
    I.estimated_error = r.est;
    I.device_ms = ms;
    I.kernel_launches = 1;
    if (want_res) {
      const double rr = B.h_rr[2 * k], bb = B.h_rr[2 * k + 1];
      I.rel_residual = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
    } else {
      I.rel_residual = -1.0;
    }
  }
  return worst;
}

int rebuild_islands(pyomgpu_ctx* c) {
  // Z of make_inv_sfc and the segment lists of line_integral from c->isl.
  const IslandSet& I = c->isl;
  std::vector<int> bi, bj;
  std::vector<int> si, sj, sd, off((size_t)I.nisle + 1, 0);
  for (int k = 1; k <= I.nisle; ++k) {
    off[k - 1] = (int)si.size();
    for (int n = 1; n <= I.nr_boundary[k - 1]; ++n) {
      const size_t o = (size_t)(k - 1) + (size_t)(n - 1) * I.nisle;
      const int i = I.boundary[o], j = I.boundary[o + (size_t)I.nisle * I.max_boundary];
      bi.push_back(i);
      bj.push_back(j);
      if (i >= 0 && i <= c->nx && j >= 0 && j <= c->ny) {  // line_integral window (streamfct_init.f90:324-332)
        const int d0 = I.line_dir[o], d1 = I.line_dir[o + (size_t)I.nisle * I.max_boundary];
        int d;
        if (d0 == 1 && d1 == 0)
          d = 0;
        else if (d0 == -1 && d1 == 0)
          d = 1;
        else if (d0 == 0 && d1 == 1)
          d = 2;
        else if (d0 == 0 && d1 == -1)
          d = 3;
        else
          return fail(PYOMGPU_EISLAND, "missing line_dir in line integral (island %d point %d)", k, n);
        si.push_back(i);
        sj.push_back(j);
        sd.push_back(d);
      }
    }
  }
  off[I.nisle] = (int)si.size();
  for (int* p : {c->bnd_i, c->bnd_j, c->idev.seg_i, c->idev.seg_j, c->idev.seg_d, c->idev.seg_off})
    if (p) cudaFree(p);
  c->bnd_i = c->bnd_j = nullptr;
  c->idev = IslandDev{};
  c->nbnd = (int)bi.size();
  if (int rc = dalloc(&c->bnd_i, bi.size())) return rc;
  if (int rc = dalloc(&c->bnd_j, bj.size())) return rc;
  if (!bi.empty()) {
    CK(cudaMemcpy(c->bnd_i, bi.data(), bi.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->bnd_j, bj.data(), bj.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  c->idev.nisle = I.nisle;
  if (int rc = dalloc(&c->idev.seg_i, si.size())) return rc;
  if (int rc = dalloc(&c->idev.seg_j, sj.size())) return rc;
  if (int rc = dalloc(&c->idev.seg_d, sd.size())) return rc;
  if (int rc = dalloc(&c->idev.seg_off, off.size())) return rc;
  if (!si.empty()) {
    CK(cudaMemcpy(c->idev.seg_i, si.data(), si.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->idev.seg_j, sj.data(), sj.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->idev.seg_d, sd.data(), sd.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(c->idev.seg_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  launch_build_inv_diag(c->g, c->sf, c->bnd_i, c->bnd_j, c->nbnd, 0);
  c->fast.op32_stale = true;  // Z changed
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  for (double* p : {c->line_forc, c->line_psi0})
    if (p) cudaFree(p);
  c->line_forc = c->line_psi0 = nullptr;
  if (int rc = dalloc(&c->line_forc, (size_t)std::max(1, I.nisle))) return rc;
  if (int rc = dalloc(&c->line_psi0, (size_t)std::max(1, I.nisle))) return rc;
  c->have_islands = true;
  return 0;
}

LineGeo line_geo(const pyomgpu_ctx* c) {
  return LineGeo{c->dxu, c->dyu, c->cost, c->cosu, c->dxt, c->dyt, c->hur, c->hvr, c->mU, c->mV};
}

int factor_line_psin(pyomgpu_ctx* c) {
  const int nisle = c->isl.nisle;
  c->lu_singular = false;
  if (nisle <= 1) return 0;
  const int m = nisle - 1;
  std::vector<double> a((size_t)m * m);
  for (int col = 0; col < m; ++col)
    for (int r = 0; r < m; ++r) a[(size_t)r + (size_t)col * m] = c->line_psin[(size_t)(r + 1) + (size_t)(col + 1) * nisle];
  std::vector<int> ipiv;
  const int info = lu_factor(m, a, ipiv);
  c->lu_singular = info != 0;
  for (double* p : {c->lu})
    if (p) cudaFree(p);
  if (c->ipiv) cudaFree(c->ipiv);
  if (int rc = dalloc(&c->lu, a.size())) return rc;
  if (int rc = dalloc(&c->ipiv, ipiv.size())) return rc;
  CK(cudaMemcpy(c->lu, a.data(), a.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->ipiv, ipiv.data(), ipiv.size() * sizeof(int), cudaMemcpyHostToDevice));
  return 0;
}

// psin solves (streamfct_init.f90:272-287) and line_psin (:292-303).
int psin_and_line_psin(pyomgpu_ctx* c, double eps, int max_it, cudaStream_t st) {
  const int nisle = c->isl.nisle;
  if (c->psin) cudaFree(c->psin);
  c->psin = nullptr;
  if (int rc = dalloc(&c->psin, c->n2 * (size_t)std::max(1, nisle))) return rc;
  c->psin_iters.assign((size_t)nisle, 0);
  int worst = 0;
  std::vector<double> init(c->n2);
  const IslandSet& I = c->isl;
  // psin(:,:,isle) = 1 on the island's perimeter, 0 elsewhere (streamfct_init.f90:274-280)
  for (int isle = 1; isle <= nisle; ++isle) {
    std::fill(init.begin(), init.end(), 0.0);
    for (int n = 1; n <= I.nr_boundary[isle - 1]; ++n) {
      const size_t o = (size_t)(isle - 1) + (size_t)(n - 1) * nisle;
      const int i = I.boundary[o], j = I.boundary[o + (size_t)nisle * I.max_boundary];
      if (i >= -1 && i <= c->nx + 2 && j >= -1 && j <= c->ny + 2) init[fidx(c->nx, i, j)] = 1.0;
    }
    CK(cudaMemcpyAsync(c->psin + (size_t)(isle - 1) * c->n2, init.data(), c->n2 * sizeof(double),
                       cudaMemcpyHostToDevice, st));
  }
  // all islands' solves (zero forcing) in one work-queue launch per chunk of at most 4 GiB of work vectors
  const size_t per = 5 * align32(c->g.size());
  const int chunk = (int)std::max<size_t>(1, ((size_t)1 << 29) / per);
  for (int k0 = 0; k0 < nisle; k0 += chunk) {
    const int k1 = std::min(nisle, k0 + chunk);
    std::vector<BatchSpec> v;
    for (int k = k0; k < k1; ++k) v.push_back(BatchSpec{c, nullptr, c->psin + (size_t)k * c->n2});
    std::vector<pyomgpu_solve_info> infos(v.size());
    const double e_k = c->psin_rtol > 0.0 ? 0.0 : eps;
    const int m_k = c->psin_rtol > 0.0 ? std::max(max_it, 1000000) : max_it;
    // on-chip solves side by side where the grid fits; the work-queue kernel otherwise
    bool resident = false;
    int rc = PYOMGPU_OK;
    if (c->batch_kernel != 1) {
      size_t work = 0;
      for (const BatchSpec& b : v) work += batch_job_words(b.c->g.size());
      if ((rc = batch_reserve(c, (int)v.size(), work, 1))) return rc;
      rc = run_res_multi(c, v, e_k, m_k, c->psin_rtol, false, infos.data(), nullptr, st, &resident,
                         c->psin_weighted);
      if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
    }
    if (!resident) {
      rc = run_batch(c, v, e_k, m_k, c->psin_rtol, false, infos.data(), nullptr, st, c->psin_weighted);
      if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
    }
    for (int k = k0; k < k1; ++k) {
      const pyomgpu_solve_info& info = infos[k - k0];
      if (info.status == PYOMGPU_NAN) return fail(PYOMGPU_NAN, "psin solve of island %d: estimated error is NaN", k + 1);
      worst = std::max(worst, info.status);
      c->psin_iters[k] = info.iterations;
    }
  }
  for (int k = 0; k < nisle; ++k) launch_setcyclic_user(c->g, c->psin + (size_t)k * c->n2, st);
  CK(cudaGetLastError());
  c->have_psin = true;
  // line_psin(n, isle) = line integral around island n of the velocity of psin(:,:,isle)
  double* dout = nullptr;
  if (int rc = dalloc(&dout, (size_t)nisle * nisle)) return rc;
  launch_line_integral_psi(c->nx, c->ny, c->idev, line_geo(c), c->psin, c->n2, nisle, 0, nisle, dout, st);
  c->line_psin.assign((size_t)nisle * nisle, 0.0);
  cudaError_t e = cudaMemcpyAsync(c->line_psin.data(), dout, sizeof(double) * nisle * nisle, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(dout);
  if (e != cudaSuccess) return fail(PYOMGPU_ECUDA, "line_psin: %s", cudaGetErrorString(e));
  c->have_line_psin = true;
  if (int rc = factor_line_psin(c)) return rc;
  return worst;
}

int island_error(int rc) {
  switch (rc) {
    case kIslMaxipp:
      return fail(PYOMGPU_EISLAND, "maxipp too small (island_module.f90:256)");
    case kIslQueue:
      return fail(PYOMGPU_EISLAND, "queue fault in qpush (island_module.f90:310): raise maxq");
    case kIslMnisle:
      return fail(PYOMGPU_EISLAND, "mnisle too small (island_module.f90:86)");
    case kIslMissing:
      return fail(PYOMGPU_EISLAND, "cannot find island in map (streamfct_init.f90:81)");
    case kIslNoStart:
      return fail(PYOMGPU_EISLAND, "found no starting point for line integral (streamfct_init.f90:162)");
    case kIslLostTrack:
      return fail(PYOMGPU_EISLAND, "unknown situation or lost track (streamfct_init.f90:224)");
    case kIslMaxBoundary:
      return fail(PYOMGPU_EISLAND, "increase max_boundary (streamfct_init.f90:252)");
    default:
      return fail(PYOMGPU_EISLAND, "island map read outside the grid");
  }
}

IslandLimits limits(int mnisle, int maxipp, int maxq) {
  IslandLimits L;
  if (mnisle > 0) L.mnisle = mnisle;
  if (maxipp > 0) L.maxipp = maxipp;
  if (maxq > 0) L.maxq = maxq;
  return L;
}

StepDev step_dev(const pyomgpu_ctx* c, const pyomgpu_state* s) {
  StepDev d{};
  d.nx = c->nx;
  d.ny = c->ny;
  d.nz = s->nz;
  d.cyclic_x = c->g.cyclic_x;
  d.cyclic_y = c->g.cyclic_y;
  d.taum1 = s->taum1;
  d.tau = s->tau;
  d.taup1 = s->taup1;
  d.dt_mom = s->dt_mom;
  d.AB_eps = s->AB_eps;
  d.grav = s->grav;
  d.rho_0 = s->rho_0;
  d.dxt = c->dxt;
  d.dxu = c->dxu;
  d.dyt = c->dyt;
  d.dyu = c->dyu;
  d.cost = c->cost;
  d.cosu = c->cosu;
  d.dzt = s->dzt;
  d.dzw = s->dzw;
  d.hur = c->hur;
  d.hvr = c->hvr;
  d.maskT = s->maskT;
  d.maskU = s->maskU;
  d.maskV = s->maskV;
  d.rho = s->rho;
  d.du_mix = s->du_mix;
  d.dv_mix = s->dv_mix;
  d.u = s->u;
  d.v = s->v;
  d.du = s->du;
  d.dv = s->dv;
  d.p_hydro = s->p_hydro;
  d.psi = s->psi;
  d.dpsi = s->dpsi;
  return d;
}

bool state_ok(const pyomgpu_state* s) {
  const void* ptrs[] = {s->dzt, s->dzw, s->maskT, s->maskU, s->maskV, s->rho, s->u, s->v, s->du, s->dv,
                        s->du_mix, s->dv_mix, s->p_hydro, s->psi, s->dpsi};
  for (const void* p : ptrs)
    if (!is_device_ptr(p)) return false;
  return s->nz >= 1 && s->tau >= 1 && s->tau <= 3 && s->taup1 >= 1 && s->taup1 <= 3 && s->taum1 >= 1 &&
         s->taum1 <= 3;
}

// island_boundaries_gpu on a host or device kbot
int gpu_islands(int nx, int ny, bool cyclic_x, const int32_t* kbot, const IslandLimits& L, IslandSet& S,
                cudaStream_t st) {
  const int32_t* kd = kbot;
  int32_t* tmp = nullptr;
  const size_t n2 = (size_t)(nx + 4) * (ny + 4);
  if (!is_device_ptr(kbot)) {
    if (int rc = dalloc(&tmp, n2)) return rc;
    if (cudaMemcpyAsync(tmp, kbot, n2 * sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess) {
      cudaFree(tmp);
      return fail(PYOMGPU_ECUDA, "island kbot upload");
    }
    kd = tmp;
  }
  const int rc = island_boundaries_gpu(nx, ny, cyclic_x, kd, L, S, nullptr, (void*)st);
  if (tmp) cudaFree(tmp);
  if (rc <= -100) return fail(PYOMGPU_ECUDA, "GPU island labelling failed (%d)", rc);
  if (rc) return island_error(rc);
  return PYOMGPU_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

int32_t pyomgpu_version(void) { return 1; }

const char* pyomgpu_last_error(void) { return g_last_error.c_str(); }

int32_t pyomgpu_ctx_create(const pyomgpu_grid* gr, pyomgpu_ctx** out) {
  if (!gr || !out) return fail(PYOMGPU_EINVAL, "null argument");
  *out = nullptr;
  if (gr->onx != 2) return fail(PYOMGPU_EINVAL, "onx must be 2 (got %d)", gr->onx);
  if (gr->nx < 4 || gr->ny < 4) return fail(PYOMGPU_EINVAL, "grid must be at least 4x4 (got %dx%d)", gr->nx, gr->ny);
  if (!gr->dxt || !gr->dxu || !gr->dyt || !gr->dyu || !gr->cost || !gr->cosu || !gr->hur || !gr->hvr)
    return fail(PYOMGPU_EINVAL, "missing grid array");
  auto* c = new pyomgpu_ctx();
  auto bail = [&](int rc) {
    delete c;
    return rc;
  };
  CK(cudaGetDevice(&c->device));
  CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
  c->nx = gr->nx;
  c->ny = gr->ny;
  c->n2 = (size_t)(c->nx + 4) * (c->ny + 4);
  c->g.nx = c->nx;
  c->g.ny = c->ny;
  c->g.pitch = ((c->nx + 4 + kXOff) + 31) / 32 * 32;
  c->g.cyclic_x = gr->enable_cyclic_x ? 1 : 0;
  c->g.cyclic_y = gr->enable_cyclic_y ? 1 : 0;
  c->free_surface = gr->enable_free_surface;
  c->grav = gr->grav;
  c->dt_mom = gr->dt_mom;
  const size_t X = c->nx + 4, Y = c->ny + 4, n2 = c->n2;
  int rc;
  if ((rc = upload(&c->dxt, gr->dxt, X)) || (rc = upload(&c->dxu, gr->dxu, X)) || (rc = upload(&c->dyt, gr->dyt, Y)) ||
      (rc = upload(&c->dyu, gr->dyu, Y)) || (rc = upload(&c->cost, gr->cost, Y)) ||
      (rc = upload(&c->cosu, gr->cosu, Y)) || (rc = upload(&c->hur, gr->hur, n2)) ||
      (rc = upload(&c->hvr, gr->hvr, n2)) || (rc = upload(&c->mU, gr->maskU_top, n2)) ||
      (rc = upload(&c->mV, gr->maskV_top, n2)))
    return bail(rc);
  c->have_sp = gr->hu && gr->hv && gr->maskT_top;
  if (c->have_sp) {
    if ((rc = upload(&c->hu, gr->hu, n2)) || (rc = upload(&c->hv, gr->hv, n2)) || (rc = upload(&c->mT, gr->maskT_top, n2)))
      return bail(rc);
  }
  const size_t P = c->g.size();
  for (OpBuf* op : {&c->sf, &c->sp}) {
    if (op == &c->sp && !c->have_sp) break;
    if ((rc = dalloc(&op->FX, P)) || (rc = dalloc(&op->FY, P)) || (rc = dalloc(&op->W, P)) ||
        (rc = dalloc(&op->ax, X)) || (rc = dalloc(&op->bx, Y)) || (rc = dalloc(&op->by, Y)))
      return bail(rc);
    if (cudaMemset(op->FX, 0, P * 8) || cudaMemset(op->FY, 0, P * 8) || cudaMemset(op->W, 0, P * 8))
      return bail(fail(PYOMGPU_ECUDA, "memset"));
  }
  GridDev gd{c->nx, c->ny, c->dxt, c->dxu, c->dyt, c->dyu, c->cost, c->cosu, c->hur, c->hvr, c->hu, c->hv, c->mT};
  launch_build_op_streamfunction(gd, c->g, c->sf, 0);
  launch_build_inv_diag(c->g, c->sf, nullptr, nullptr, 0, 0);
  if (c->have_sp) {
    launch_build_op_surf_press(gd, c->g, c->sp, 0);
    c->sp.dcoef = c->free_surface ? -1.0 / (c->grav * (c->dt_mom * c->dt_mom)) : 0.0;
  }
  if ((rc = dalloc(&c->res, P)) || (rc = dalloc(&c->s0, P)) || (rc = dalloc(&c->s1, P)) || (rc = dalloc(&c->As, P)) ||
      (rc = dalloc(&c->sol, P)) || (rc = dalloc(&c->stage_a, n2)) || (rc = dalloc(&c->stage_b, n2)) ||
      (rc = dalloc(&c->fpx, n2)) || (rc = dalloc(&c->fpy, n2)) || (rc = dalloc(&c->forc, n2)) ||
      (rc = dalloc(&c->zeros, n2)) || (rc = dalloc(&c->part, 2 * 4096)) || (rc = dalloc(&c->scal, 16)))
    return bail(rc);
  if (cudaMemset(c->zeros, 0, n2 * 8) || cudaMemset(c->sol, 0, P * 8) || cudaMemset(c->As, 0, P * 8))
    return bail(fail(PYOMGPU_ECUDA, "memset"));
  int per_sm = 0;
  for (bool sp : {false, true})
    if (cudaFuncSetAttribute(cg_ref_kernel_ptr(sp), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kCGSmemMax) != cudaSuccess)
      return bail(fail(PYOMGPU_ECUDA, "cannot reserve %zu bytes of shared memory", kCGSmemMax));
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_ref_kernel_ptr(false), kCGThreads, kCGSmem) !=
          cudaSuccess ||
      per_sm < 1)
    return bail(fail(PYOMGPU_ECUDA, "occupancy query failed"));
  int per_sm2 = per_sm;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, cg_ref_kernel_ptr(true), kCGThreads, kCGSmem);
  c->max_blocks = std::min(per_sm, std::max(1, per_sm2)) * c->nsm;
  if ((rc = dalloc((double**)&c->ctl, 2)) || (rc = dalloc(&c->slots, (size_t)2 * c->max_blocks * 4)) ||
      (rc = dalloc((double**)&c->d_result, 4)))
    return bail(rc);
  if (cudaMallocHost((void**)&c->h_result, sizeof(CGResult)) != cudaSuccess ||
      cudaMallocHost((void**)&c->h_scal, 64) != cudaSuccess)
    return bail(fail(PYOMGPU_ENOMEM, "cudaMallocHost"));
  if (cudaEventCreate(&c->e0) != cudaSuccess || cudaEventCreate(&c->e1) != cudaSuccess)
    return bail(fail(PYOMGPU_ECUDA, "event create"));
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return bail(fail(PYOMGPU_ECUDA, "ctx build: %s", cudaGetErrorString(e)));
  *out = c;
  return PYOMGPU_OK;
}

void pyomgpu_ctx_destroy(pyomgpu_ctx* c) { delete c; }

int32_t pyomgpu_set_sync_timeout(pyomgpu_ctx* c, double seconds) {
  if (!c || !(seconds > 0)) return fail(PYOMGPU_EINVAL, "bad timeout");
  c->timeout_s = seconds;
  return PYOMGPU_OK;
}

int32_t pyomgpu_inject_barrier_stall(pyomgpu_ctx* c, int32_t enable) {
  if (!c) return fail(PYOMGPU_EINVAL, "null context");
  c->stall_next = enable ? 1u : 0u;
  return PYOMGPU_OK;
}

int32_t pyomgpu_set_cg_kernel(pyomgpu_ctx* c, int32_t kernel) {
  if (!c || kernel < 0 || kernel > 3) return fail(PYOMGPU_EINVAL, "set_cg_kernel: bad arguments");
  if (kernel >= 2) {
    if (int rc = res_plan(c)) return rc;
    if (!c->resd.ok) return fail(PYOMGPU_EINVAL, "the grid does not fit the resident kernel");
  }
  c->cg_kernel = kernel;
  return PYOMGPU_OK;
}

int32_t pyomgpu_plan_batch(int32_t nsm, int32_t count, const int32_t* blocks, const double* est, int32_t tries,
                           int32_t* rank, double* start, int32_t* gang, double* makespan) {
  if (nsm < 1 || count < 1 || !blocks || !est || tries < 0) return fail(PYOMGPU_EINVAL, "plan_batch: bad arguments");
  std::vector<int> nb((size_t)count);
  std::vector<double> e((size_t)count);
  for (int k = 0; k < count; ++k) {
    if (blocks[k] < 1 || blocks[k] > nsm || !(est[k] >= 0.0)) return fail(PYOMGPU_EINVAL, "plan_batch: job %d", k);
    nb[k] = blocks[k];
    e[k] = est[k];
  }
  GangPlan plan;
  plan_gangs(nsm, nb, e, nullptr, tries, plan);
  for (int k = 0; k < count; ++k) {
    if (rank) rank[k] = plan.rank[k];
    if (start) start[k] = plan.start[k];
    if (gang)
      for (int q = 0; q < nsm; ++q) gang[(size_t)k * nsm + q] = q < nb[k] ? plan.gang[k][q] : -1;
  }
  if (makespan) *makespan = plan.makespan;
  return PYOMGPU_OK;
}

int32_t pyomgpu_plan_cut(int32_t nx, int32_t ny, int32_t max_blocks, int64_t smem_cap, int32_t points_per_thread,
                         int32_t least_block_time, int32_t fp32, int32_t* out, double* est_ns) {
  const int p = points_per_thread;
  const bool p_ok = fp32 ? (p == 0 || p == 16 || p == 32) : (p == 0 || p == 4 || p == 8 || p == 16);
  if (nx < 2 || ny < 2 || max_blocks < 1 || max_blocks >= kResMaxSlots || smem_cap < 0 || !out || !p_ok)
    return fail(PYOMGPU_EINVAL, "plan_cut: bad arguments");
  ResCut cut;
  const bool ok = res_cut(nx, ny, max_blocks, (size_t)smem_cap, p, least_block_time != 0, cut, fp32 != 0);
  out[0] = ok ? cut.npx : 0;
  out[1] = ok ? cut.npy : 0;
  out[2] = ok ? cut.w : 0;
  out[3] = ok ? cut.h : 0;
  out[4] = ok ? cut.p : 0;
  if (est_ns) *est_ns = ok ? cut.cost : 0.0;
  return PYOMGPU_OK;
}

int32_t pyomgpu_batch_schedule(pyomgpu_ctx* c, int32_t count, double* start_ms, double* end_ms, int32_t* blocks) {
  if (!c || count < 0) return fail(PYOMGPU_EINVAL, "batch_schedule: bad arguments");
  if ((int)c->sched_start.size() != count)
    return fail(PYOMGPU_ESTATE, "batch_schedule: the last resident batch of this context had %d solves",
                (int)c->sched_start.size());
  for (int k = 0; k < count; ++k) {
    if (start_ms) start_ms[k] = c->sched_start[k];
    if (end_ms) end_ms[k] = c->sched_end[k];
    if (blocks) blocks[k] = c->sched_blocks[k];
  }
  return PYOMGPU_OK;
}

int32_t pyomgpu_set_batch_kernel(pyomgpu_ctx* c, int32_t kernel) {
  if (!c || kernel < 0 || kernel > 2) return fail(PYOMGPU_EINVAL, "set_batch_kernel: bad arguments");
  c->batch_kernel = kernel;
  return PYOMGPU_OK;
}

int32_t pyomgpu_resident_layout(pyomgpu_ctx* c, int32_t* npx, int32_t* npy, int32_t* points_per_thread) {
  if (!c) return fail(PYOMGPU_EINVAL, "null context");
  if (int rc = res_plan(c)) return rc;
  if (!c->resd.ok) return fail(PYOMGPU_EINVAL, "the grid does not fit the resident kernel");
  if (npx) *npx = c->resd.npx;
  if (npy) *npy = c->resd.npy;
  if (points_per_thread) *points_per_thread = c->resd.p;
  return PYOMGPU_OK;
}

int32_t pyomgpu_resident_layout32(pyomgpu_ctx* c, int32_t* npx, int32_t* npy, int32_t* points_per_thread) {
  if (!c) return fail(PYOMGPU_EINVAL, "null context");
  if (int rc = res_plan32(c)) return rc;
  if (!c->resd.ok32) return fail(PYOMGPU_EINVAL, "the grid does not fit the FP32 resident kernel");
  if (npx) *npx = c->resd.npx32;
  if (npy) *npy = c->resd.npy32;
  if (points_per_thread) *points_per_thread = c->resd.p32;
  return PYOMGPU_OK;
}

int32_t pyomgpu_set_psin_solve(pyomgpu_ctx* c, double rtol, int32_t weighted) {
  if (!c || rtol < 0.0 || rtol >= 1.0 || (weighted != 0 && weighted != 1))
    return fail(PYOMGPU_EINVAL, "set_psin_solve: bad arguments");
  c->psin_rtol = rtol;
  c->psin_weighted = weighted;
  return PYOMGPU_OK;
}

int32_t pyomgpu_resident_trace(pyomgpu_ctx* c, const double* forc, double* sol, double rtol, int32_t it0,
                               int32_t nit, uint64_t* out, int32_t* nblocks, pyomgpu_solve_info* info,
                               pyomgpu_stream stream) {
  if (!c || !out || it0 < 0 || nit < 1 || nit > 4096) return fail(PYOMGPU_EINVAL, "resident trace: bad arguments");
  if (int rc = res_plan(c)) return rc;
  if (!c->resd.ok) return fail(PYOMGPU_EINVAL, "the grid does not fit the resident kernel");
  auto& R = c->resd;
  const int nb = R.npx * R.npy;
  const size_t words = (size_t)nb * nit * kResTracePhases;
  if (words > R.trace_cap) {
    if (R.trace) cudaFree(R.trace);
    R.trace = nullptr;
    R.trace_cap = 0;
    if (int rc = dalloc(&R.trace, words)) return rc;
    R.trace_cap = words;
  }
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(R.trace, 0, words * sizeof(uint64_t), st));
  const int saved = c->cg_kernel;
  c->cg_kernel = 2;
  R.trace_it0 = it0;
  R.trace_nit = nit;
  const int rc = pyomgpu_solve_rtol(c, forc, sol, rtol, PYOMGPU_PREC_F64, 1000000, info, stream);
  R.trace_nit = 0;
  c->cg_kernel = saved;
  if (rc != PYOMGPU_OK && rc != PYOMGPU_MAXITER) return rc;
  CK(cudaMemcpyAsync(out, R.trace, words * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (nblocks) *nblocks = nb;
  return rc;
}

int32_t pyomgpu_autotune(pyomgpu_ctx* c, int32_t iterations, int32_t* tile_x, int32_t* tile_y, int32_t* grid,
                         double* us_per_iteration, pyomgpu_stream stream) {
  if (!c || iterations < 10) return fail(PYOMGPU_EINVAL, "autotune: bad arguments");
  if (!c->have_islands) return fail(PYOMGPU_ESTATE, "autotune: set up the islands first");
  cudaStream_t st = (cudaStream_t)stream;
  launch_fill_pseudorandom(c->stage_a, c->n2, 12345u, st);  // a fixed right-hand side with all scales
  const size_t bytes = c->g.size() * sizeof(double);
  struct Cand {
    int tx, ty, grid;
  };
  std::vector<Cand> cands;
  for (int tx : {32, 64, 96, 128})
    for (int ty : {8, 16, 24, 32}) {
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_ref_kernel_ptr(false), kCGThreads,
                                                        cg_smem_bytes(tx, ty)) != cudaSuccess ||
          per_sm < 1)
        continue;
      const int maxb = std::min(per_sm * c->nsm, c->max_blocks);
      const int ntiles = ((c->nx + tx - 1) / tx) * ((c->ny + ty - 1) / ty);
      const int g1 = std::min(maxb, ntiles);
      cands.push_back({tx, ty, g1});
      const int per = (ntiles + maxb - 1) / maxb;  // tiles of the busiest block
      const int g2 = (ntiles + per - 1) / per;     // fewest blocks with the same busiest load
      if (g2 != g1 && g2 >= 1) cands.push_back({tx, ty, g2});
    }
  pyomgpu_ctx::Tune best{};
  best.us_per_it = 1e300;
  const int kernel_choice = c->cg_kernel;
  c->cg_kernel = 1;  // the tiled kernel is the one tuned
  for (int pass = 0; pass < 2; ++pass)  // every candidate twice, the faster run counts
    for (const Cand& k : cands) {
      c->tune = pyomgpu_ctx::Tune{true, k.tx, k.ty, k.grid, 0.0};
      CK(cudaMemsetAsync(c->sol, 0, bytes, st));
      pyomgpu_solve_info info{};
      int rc = run_cg_ref(c, false, c->stage_a, 0.0, iterations, 0.0, &info, st);
      if (rc < 0 || rc == PYOMGPU_TIMEOUT) {
        c->tune = pyomgpu_ctx::Tune{};
        c->cg_kernel = kernel_choice;
        return rc;
      }
      if (info.iterations < 1) continue;
      const double us = 1e3 * info.device_ms / info.iterations;
      if (us < best.us_per_it) best = pyomgpu_ctx::Tune{true, k.tx, k.ty, k.grid, us};
    }
  c->tune = best.done ? best : pyomgpu_ctx::Tune{};
  c->cg_kernel = kernel_choice;
  if (tile_x) *tile_x = c->tune.done ? c->tune.tx : kTileX;
  if (tile_y) *tile_y = c->tune.done ? c->tune.ty : kTileY;
  if (grid) *grid = c->tune.grid;
  if (us_per_iteration) *us_per_iteration = c->tune.us_per_it;
  return PYOMGPU_OK;
}

int32_t pyomgpu_island_boundaries(int32_t nx, int32_t ny, int32_t cyclic_x, const int32_t* kbot, int32_t mnisle,
                                  int32_t maxipp, int32_t maxq, int32_t* nisle, int32_t* max_boundary,
                                  int32_t* boundary, int32_t* line_dir, int32_t* nr_boundary) {
  if (!kbot || !nisle || !max_boundary || nx < 4 || ny < 4) return fail(PYOMGPU_EINVAL, "bad arguments");
  IslandLimits L = limits(mnisle, maxipp, maxq);
  std::vector<int> allmap;
  int n = 0, mb = 0;
  int rc = island_map(nx, ny, cyclic_x != 0, kbot, L, allmap, &n, &mb);
  if (rc) return island_error(rc);
  if (!boundary) {
    *nisle = n;
    *max_boundary = mb;
    return PYOMGPU_OK;
  }
  if (*nisle != n || *max_boundary != mb || !line_dir || !nr_boundary)
    return fail(PYOMGPU_EINVAL, "island arrays sized for (%d,%d), need (%d,%d)", *nisle, *max_boundary, n, mb);
  IslandSet S;
  rc = island_trace(nx, ny, cyclic_x != 0, allmap, n, mb, L, S);
  if (rc) return island_error(rc);
  std::copy(S.boundary.begin(), S.boundary.end(), boundary);
  std::copy(S.line_dir.begin(), S.line_dir.end(), line_dir);
  std::copy(S.nr_boundary.begin(), S.nr_boundary.end(), nr_boundary);
  return PYOMGPU_OK;
}

int32_t pyomgpu_island_boundaries_gpu(int32_t nx, int32_t ny, int32_t cyclic_x, const int32_t* kbot, int32_t mnisle,
                                      int32_t maxipp, int32_t maxq, int32_t* nisle, int32_t* max_boundary,
                                      int32_t* boundary, int32_t* line_dir, int32_t* nr_boundary,
                                      pyomgpu_stream stream) {
  if (!kbot || !nisle || !max_boundary || nx < 4 || ny < 4) return fail(PYOMGPU_EINVAL, "bad arguments");
  IslandLimits L = limits(mnisle, maxipp, maxq);
  IslandSet S;
  if (int rc = gpu_islands(nx, ny, cyclic_x != 0, kbot, L, S, (cudaStream_t)stream)) return rc;
  if (!boundary) {
    *nisle = S.nisle;
    *max_boundary = S.max_boundary;
    return PYOMGPU_OK;
  }
  if (*nisle != S.nisle || *max_boundary != S.max_boundary || !line_dir || !nr_boundary)
    return fail(PYOMGPU_EINVAL, "island arrays sized for (%d,%d), need (%d,%d)", *nisle, *max_boundary, S.nisle,
                S.max_boundary);
  std::copy(S.boundary.begin(), S.boundary.end(), boundary);
  std::copy(S.line_dir.begin(), S.line_dir.end(), line_dir);
  std::copy(S.nr_boundary.begin(), S.nr_boundary.end(), nr_boundary);
  return PYOMGPU_OK;
}

int32_t pyomgpu_isleperim(const int32_t* kmt, int32_t imt, int32_t jmt, int32_t cyclic, int32_t mnisle,
                          int32_t maxipp, int32_t maxq, int32_t* map, int32_t* nisle, int32_t* nippts) {
  if (!kmt || !map || !nisle || imt < 3 || jmt < 3) return fail(PYOMGPU_EINVAL, "bad isleperim arguments");
  IslandLimits L = limits(mnisle, maxipp, maxq);
  std::vector<int> np;
  int rc = pyomgpu::isleperim(kmt, imt, jmt, cyclic != 0, L, map, nisle, &np);
  if (rc) return island_error(rc);
  if (nippts) std::copy(np.begin(), np.end(), nippts);
  return PYOMGPU_OK;
}

int32_t pyomgpu_streamfunction_init(pyomgpu_ctx* c, const int32_t* kbot, int32_t mnisle, int32_t maxipp, int32_t maxq,
                                    double eps, int32_t max_it, pyomgpu_stream stream) {
  if (!c || !kbot) return fail(PYOMGPU_EINVAL, "null argument");
  if (c->g.cyclic_y)  // streamfct_init.f90:27-30
    return fail(PYOMGPU_EINVAL, "cyclic meridional boundary conditions not implemented for the streamfunction");
  cudaStream_t st = (cudaStream_t)stream;
  IslandLimits L = limits(mnisle, maxipp, maxq);
  IslandSet S;
  int rc = gpu_islands(c->nx, c->ny, c->g.cyclic_x != 0, kbot, L, S, st);  // labelling + tracing on the GPU
  if (rc) return rc;
  c->isl = std::move(S);
  if ((rc = rebuild_islands(c))) return rc;
  return psin_and_line_psin(c, eps, max_it, st);
}

int32_t pyomgpu_island_sizes(pyomgpu_ctx* c, int32_t* nisle, int32_t* max_boundary) {
  if (!c || !c->have_islands) return fail(PYOMGPU_ESTATE, "no islands set");
  if (nisle) *nisle = c->isl.nisle;
  if (max_boundary) *max_boundary = c->isl.max_boundary;
  return PYOMGPU_OK;
}

int32_t pyomgpu_get_islands(pyomgpu_ctx* c, int32_t* boundary, int32_t* line_dir, int32_t* nr_boundary, double* psin,
                            double* line_psin, int32_t* psin_iterations, pyomgpu_stream stream) {
  if (!c || !c->have_islands) return fail(PYOMGPU_ESTATE, "no islands set");
  const IslandSet& I = c->isl;
  if (boundary) std::copy(I.boundary.begin(), I.boundary.end(), boundary);
  if (line_dir) std::copy(I.line_dir.begin(), I.line_dir.end(), line_dir);
  if (nr_boundary) std::copy(I.nr_boundary.begin(), I.nr_boundary.end(), nr_boundary);
  if (psin_iterations && !c->psin_iters.empty()) std::copy(c->psin_iters.begin(), c->psin_iters.end(), psin_iterations);
  if (line_psin && c->have_line_psin) std::copy(c->line_psin.begin(), c->line_psin.end(), line_psin);
  if (psin && c->have_psin) {
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = c->n2 * (size_t)I.nisle * sizeof(double);
    CK(cudaMemcpyAsync(psin, c->psin, bytes, cudaMemcpyDefault, st));
    CK(cudaStreamSynchronize(st));
  }
  return PYOMGPU_OK;
}

int32_t pyomgpu_set_islands(pyomgpu_ctx* c, const pyomgpu_islands* isl, const double* psin, const double* line_psin,
                            pyomgpu_stream stream) {
  if (!c || !isl || isl->nisle < 0 || (isl->nisle > 0 && (!isl->boundary || !isl->line_dir || !isl->nr_boundary)))
    return fail(PYOMGPU_EINVAL, "bad island description");
  IslandSet S;
  S.nisle = isl->nisle;
  S.max_boundary = isl->max_boundary;
  const size_t nb = (size_t)isl->nisle * isl->max_boundary * 2;
  S.boundary.assign(isl->boundary, isl->boundary + nb);
  S.line_dir.assign(isl->line_dir, isl->line_dir + nb);
  S.nr_boundary.assign(isl->nr_boundary, isl->nr_boundary + isl->nisle);
  for (int k = 0; k < S.nisle; ++k)
    if (S.nr_boundary[k] < 0 || S.nr_boundary[k] > S.max_boundary)
      return fail(PYOMGPU_EINVAL, "nr_boundary(%d) out of range", k + 1);
  c->isl = std::move(S);
  c->have_psin = c->have_line_psin = false;
  int rc = rebuild_islands(c);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (psin) {
    if (c->psin) cudaFree(c->psin);
    c->psin = nullptr;
    if ((rc = dalloc(&c->psin, c->n2 * (size_t)std::max(1, c->isl.nisle)))) return rc;
    CK(cudaMemcpyAsync(c->psin, psin, c->n2 * (size_t)c->isl.nisle * sizeof(double), cudaMemcpyDefault, st));
    CK(cudaStreamSynchronize(st));
    c->have_psin = true;
  }
  if (line_psin) {
    c->line_psin.assign(line_psin, line_psin + (size_t)c->isl.nisle * c->isl.nisle);
    c->have_line_psin = true;
    if ((rc = factor_line_psin(c))) return rc;
  }
  return PYOMGPU_OK;
}

int32_t pyomgpu_congrad_streamfunction(pyomgpu_ctx* c, const double* forc, double* sol, double eps, int32_t max_it,
                                       pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!c || !forc || !sol) return fail(PYOMGPU_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const double* f = nullptr;
  if (int rc = stage_in(c, forc, c->stage_a, &f, st)) return rc;
  const bool sol_dev = is_device_ptr(sol);
  const double* s_in = sol;
  if (!sol_dev) {
    CK(cudaMemcpyAsync(c->stage_b, sol, c->n2 * sizeof(double), cudaMemcpyHostToDevice, st));
    s_in = c->stage_b;
  }
  launch_pack(c->g, s_in, c->sol, true, st);  // setcyclic_xy(sol), solve_streamfct.f90:191-192
  int rc = run_cg_ref(c, false, f, eps, max_it, 0.0, info, st);
  if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
  if (sol_dev) {
    launch_unpack(c->g, c->sol, sol, false, false, false, st);
  } else {
    launch_unpack(c->g, c->sol, c->stage_b, false, false, false, st);
    CK(cudaMemcpyAsync(sol, c->stage_b, c->n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return rc;
}

int32_t pyomgpu_congrad_streamfunction_batch(pyomgpu_ctx* const* ctx, int32_t count, const double* const* forc,
                                             double* const* sol, double eps, int32_t max_it, double rtol,
                                             pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!ctx || count < 1 || !sol) return fail(PYOMGPU_EINVAL, "bad batch arguments");
  if (!(rtol >= 0.0)) return fail(PYOMGPU_EINVAL, "rtol must be >= 0");
  for (int k = 0; k < count; ++k) {
    if (!ctx[k] || !sol[k]) return fail(PYOMGPU_EINVAL, "null context or solution in batch entry %d", k);
    if (ctx[k]->device != ctx[0]->device) return fail(PYOMGPU_EINVAL, "batch contexts on different devices");
  }
  cudaStream_t st = (cudaStream_t)stream;
  pyomgpu_ctx* o = ctx[0];
  // host arrays are staged in the tail of the owner's pool, after the solve buffers
  size_t work = 0, stage = 0;
  std::vector<char> f_host(count), s_host(count);
  for (int k = 0; k < count; ++k) {
    work += batch_job_words(ctx[k]->g.size());
    f_host[k] = forc && forc[k] && !is_device_ptr(forc[k]);
    s_host[k] = !is_device_ptr(sol[k]);
    stage += (f_host[k] + s_host[k]) * align32(ctx[k]->n2);
  }
  size_t tasks = 0;
  for (int k = 0; k < count; ++k)
    tasks += (size_t)((ctx[k]->nx + kTileX - 1) / kTileX) * ((ctx[k]->ny + kTileY - 1) / kTileY);
  if (int rc = batch_reserve(o, count, work + stage, tasks)) return rc;
  std::vector<BatchSpec> v(count);
  double* cur = o->batch.pool + work;
  for (int k = 0; k < count; ++k) {
    pyomgpu_ctx* c = ctx[k];
    v[k].c = c;
    v[k].forc = forc ? forc[k] : nullptr;
    v[k].sol = sol[k];
    if (f_host[k]) {
      CK(cudaMemcpyAsync(cur, forc[k], c->n2 * sizeof(double), cudaMemcpyHostToDevice, st));
      v[k].forc = cur;
      cur += align32(c->n2);
    }
    if (s_host[k]) {
      CK(cudaMemcpyAsync(cur, sol[k], c->n2 * sizeof(double), cudaMemcpyHostToDevice, st));
      v[k].sol = cur;
      cur += align32(c->n2);
    }
  }
  std::vector<pyomgpu_solve_info> tmp;
  if (!info) {
    tmp.resize(count);
    info = tmp.data();
  }
  bool resident = false;
  int rc = PYOMGPU_OK;
  if (o->batch_kernel != 1) {
    rc = run_res_multi(o, v, eps, max_it, rtol, rtol > 0.0, info, nullptr, st, &resident);
    if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
    if (!resident && o->batch_kernel == 2) return fail(PYOMGPU_EINVAL, "a batch grid does not fit on chip");
  }
  if (!resident) {
    rc = run_batch(o, v, eps, max_it, rtol, rtol > 0.0, info, nullptr, st);
    if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
  }
  for (int k = 0; k < count; ++k) {
    if (s_host[k]) CK(cudaMemcpyAsync(sol[k], v[k].sol, ctx[k]->n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    // the whole call: the solve launches, pack + unpack per solve (+ halo fill and 2-pass residual)
    info[k].kernel_launches += count * (rtol > 0.0 ? 5 : 2);
  }
  CK(cudaStreamSynchronize(st));
  return rc;
}

int32_t pyomgpu_congrad_surf_press(pyomgpu_ctx* c, const double* forc, double* psi, double eps, int32_t max_it,
                                   pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!c || !forc || !psi) return fail(PYOMGPU_EINVAL, "null argument");
  if (!c->have_sp) return fail(PYOMGPU_ESTATE, "context has no surface-pressure operator (hu/hv/maskT_top)");
  cudaStream_t st = (cudaStream_t)stream;
  const double* f = nullptr;
  if (int rc = stage_in(c, forc, c->stage_a, &f, st)) return rc;
  const bool dev = is_device_ptr(psi);
  const double* p_in = psi;
  if (!dev) {
    CK(cudaMemcpyAsync(c->stage_b, psi, c->n2 * sizeof(double), cudaMemcpyHostToDevice, st));
    p_in = c->stage_b;
  }
  launch_pack(c->g, p_in, c->sol, false, st);
  int rc = run_cg_ref(c, true, f, eps, max_it, 0.0, info, st);
  if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
  if (dev) {
    launch_unpack(c->g, c->sol, psi, false, false, false, st);
  } else {
    launch_unpack(c->g, c->sol, c->stage_b, false, false, false, st);
    CK(cudaMemcpyAsync(psi, c->stage_b, c->n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return rc;
}

int32_t pyomgpu_solve_rtol(pyomgpu_ctx* c, const double* forc, double* sol, double rtol, int32_t precision,
                           int32_t max_it, pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!c || !forc || !sol || !(rtol > 0) || max_it < 1) return fail(PYOMGPU_EINVAL, "bad arguments");
  if (precision != PYOMGPU_PREC_F64 && precision != PYOMGPU_PREC_F32)
    return fail(PYOMGPU_EINVAL, "precision %d not available", precision);
  const bool f32 = precision == PYOMGPU_PREC_F32;
  cudaStream_t st = (cudaStream_t)stream;
  const double* f = nullptr;
  if (int rc = stage_in(c, forc, c->stage_a, &f, st)) return rc;
  const bool dev = is_device_ptr(sol);
  const double* s_in = sol;
  if (!dev) {
    CK(cudaMemcpyAsync(c->stage_b, sol, c->n2 * sizeof(double), cudaMemcpyHostToDevice, st));
    s_in = c->stage_b;
  }
  launch_pack(c->g, s_in, c->sol, true, st);
  if (int rc = fast_setup(c, f32, st)) return rc;
  pyomgpu_solve_info tmp{};
  pyomgpu_solve_info* I = info ? info : &tmp;
  auto& F = c->fast;
  int rc = PYOMGPU_OK;
  I->iterations = 0;
  I->outer_iterations = 0;
  I->device_ms = 0.0;
  I->estimated_error = 0.0;
  if (!f32) {
    // FP64 Jacobi-PCG: the reference algorithm (two-barrier tile kernel) with
    // the residual stop
    rc = run_cg_ref(c, false, f, 0.0, max_it, rtol, I, st);
    if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
    I->kernel_launches = 6;  // pack, cg_ref, fill_cyclic, residual x2, unpack
  } else {
    I->kernel_launches = 5;  // pack, final fill_cyclic + residual x2, unpack (+6 per refinement below)
    // FP32 PCG (FP64 products) for the correction, FP64 true residual outside:
    // on the FP32 resident kernel where the grid fits on chip, else the
    // pipelined tile kernel
    if (int prc = res_plan32(c)) return prc;
    const bool use_res32 = c->cg_kernel != 1 && c->resd.ok32;
    const double inner_rtol = 1e-6;
    const int max_outer = 12;
    rc = PYOMGPU_MAXITER;
    for (int outer = 0; outer <= max_outer; ++outer) {
      launch_fill_cyclic(c->g, c->sol, st);
      launch_residual(c->g, c->sf.dev(), f, c->sol, c->part, 1024, c->scal, st);
      I->kernel_launches += 3;
      CK(cudaMemcpyAsync(c->h_scal, c->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      const double rr = c->h_scal[0], bb = c->h_scal[1];
      if (!(rr == rr)) {
        rc = PYOMGPU_NAN;
        break;
      }
      if (rr <= rtol * rtol * bb) {
        rc = PYOMGPU_OK;
        break;
      }
      if (outer == max_outer || I->iterations >= max_it) break;
      const double s = 1.0 / std::sqrt(rr);
      launch_residual_f32(c->g, c->sf.dev(), f, c->sol, s, F.b32, st);
      CK(cudaMemsetAsync(F.x32, 0, c->g.size() * sizeof(float), st));
      PipeResult R{};
      float ms = 0.f;
      const int left = std::max(1, max_it - I->iterations);
      int irc = use_res32 ? run_cg_res32(c, F.op32, F.b32, F.x32, inner_rtol, left, &R, &ms, st)
                          : run_pipe<float>(c, F.op32, F.b32, F.x32, F.r32, F.q32, F.w32, inner_rtol, left, &R, &ms,
                                            st);
      if (irc) return irc;
      I->iterations += R.iterations;
      I->outer_iterations += 1;
      I->device_ms += ms;
      I->kernel_launches += 3;  // residual_f32, cg_pipe<float>, add_correction
      if (R.status == PYOMGPU_NAN) {
        rc = PYOMGPU_NAN;
        break;
      }
      launch_add_correction(c->g, c->sol, F.x32, 1.0 / s, st);
    }
    I->status = rc;
  }
  I->converged = rc == PYOMGPU_OK;
  launch_fill_cyclic(c->g, c->sol, st);  // the border exchange that follows a solve
  launch_residual(c->g, c->sf.dev(), f, c->sol, c->part, 1024, c->scal, st);
  CK(cudaMemcpyAsync(c->h_scal, c->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (dev) {
    launch_unpack(c->g, c->sol, sol, false, false, false, st);
  } else {
    launch_unpack(c->g, c->sol, c->stage_b, false, false, false, st);
    CK(cudaMemcpyAsync(sol, c->stage_b, c->n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  const double rr = c->h_scal[0], bb = c->h_scal[1];
  I->rel_residual = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
  return rc;
}

int32_t pyomgpu_apply_op(pyomgpu_ctx* c, int32_t op, const double* p, double* res, pyomgpu_stream stream) {
  if (!c || !p || !res) return fail(PYOMGPU_EINVAL, "null argument");
  if (op == PYOMGPU_OP_SURF_PRESS && !c->have_sp) return fail(PYOMGPU_ESTATE, "no surface-pressure operator");
  if (op != PYOMGPU_OP_STREAMFUNCTION && op != PYOMGPU_OP_SURF_PRESS) return fail(PYOMGPU_EINVAL, "unknown operator");
  cudaStream_t st = (cudaStream_t)stream;
  const double* pin = nullptr;
  if (int rc = stage_in(c, p, c->stage_a, &pin, st)) return rc;
  const OpBuf& o = op == PYOMGPU_OP_SURF_PRESS ? c->sp : c->sf;
  if (is_device_ptr(res)) {
    launch_apply_op_user(c->g, o.dev(), pin, res, c->As, st);
  } else {
    launch_apply_op_user(c->g, o.dev(), pin, c->stage_b, c->As, st);
    CK(cudaMemcpyAsync(res, c->stage_b, c->n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return PYOMGPU_OK;
}

int32_t pyomgpu_get_inv_diag(pyomgpu_ctx* c, double* Z, pyomgpu_stream stream) {
  if (!c || !Z) return fail(PYOMGPU_EINVAL, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (is_device_ptr(Z)) {
    launch_unpack(c->g, c->sf.W, Z, false, false, true, st);
  } else {
    launch_unpack(c->g, c->sf.W, c->stage_b, false, false, true, st);
    CK(cudaMemcpyAsync(Z, c->stage_b, c->n2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return PYOMGPU_OK;
}

int32_t pyomgpu_line_integral(pyomgpu_ctx* c, int32_t isle, const double* uloc, const double* vloc, double* line,
                              pyomgpu_stream stream) {
  if (!c || !uloc || !vloc || !line) return fail(PYOMGPU_EINVAL, "null argument");
  if (!c->have_islands) return fail(PYOMGPU_ESTATE, "no islands set");
  if (isle < 1 || isle > c->isl.nisle) return fail(PYOMGPU_EINVAL, "island %d out of range", isle);
  cudaStream_t st = (cudaStream_t)stream;
  const double *u = nullptr, *v = nullptr;
  if (int rc = stage_in(c, uloc, c->stage_a, &u, st)) return rc;
  if (int rc = stage_in(c, vloc, c->stage_b, &v, st)) return rc;
  launch_line_integral_uv(c->nx, c->idev, line_geo(c), u, v, isle - 1, 1, c->scal, st);
  CK(cudaMemcpyAsync(c->h_scal, c->scal, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *line = c->h_scal[0];
  return PYOMGPU_OK;
}

int32_t pyomgpu_solve_streamfunction(pyomgpu_ctx* c, pyomgpu_state* s, pyomgpu_solve_info* info,
                                     pyomgpu_stream stream) {
  if (!c || !s) return fail(PYOMGPU_EINVAL, "null argument");
  if (!state_ok(s)) return fail(PYOMGPU_EINVAL, "state arrays must be device pointers with valid time levels");
  if (!c->have_islands) return fail(PYOMGPU_ESTATE, "islands not set up (streamfunction_init)");
  const int nisle = c->isl.nisle;
  if (nisle > 1 && (!c->have_psin || !c->have_line_psin)) return fail(PYOMGPU_ESTATE, "psin / line_psin missing");
  if (nisle > 1 && !is_device_ptr(s->dpsin)) return fail(PYOMGPU_EINVAL, "dpsin must be a device pointer");
  cudaStream_t st = (cudaStream_t)stream;
  StepDev d = step_dev(c, s);
  const size_t n2 = c->n2;
  launch_hydrostatic(d, st);
  launch_sf_forcing(d, c->fpx, c->fpy, c->forc, st);
  double* dp1 = s->dpsi + (size_t)(s->taup1 - 1) * n2;
  launch_first_guess(c->g, dp1, s->dpsi + (size_t)(s->tau - 1) * n2, s->dpsi + (size_t)(s->taum1 - 1) * n2, st);
  launch_pack(c->g, dp1, c->sol, true, st);
  pyomgpu_solve_info tmp{};
  pyomgpu_solve_info* I = info ? info : &tmp;
  int rc = run_cg_ref(c, false, c->forc, s->congr_epsilon, s->congr_max_iterations, 0.0, I, st);
  if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
  s->congr_itts = I->iterations;
  launch_unpack(c->g, c->sol, dp1, true, false, false, st);  // + border_exchg/setcyclic (:58-59)
  if (nisle > 1) {
    if (c->lu_singular) return fail(PYOMGPU_SINGULAR, "in solve_streamfunction, lapack info not zero");
    LineGeo lg = line_geo(c);
    launch_line_integral_uv(c->nx, c->idev, lg, c->fpx, c->fpy, 1, nisle - 1, c->line_forc, st);
    launch_line_integral_psi(c->nx, c->ny, c->idev, lg, dp1, n2, 1, 1, nisle - 1, c->line_psi0, st);
    launch_island_solve(nisle, c->lu, c->ipiv, c->line_forc, c->line_psi0, s->dpsin, s->tau, st);
  }
  launch_sf_psi_update(d, c->psin, nisle, s->dpsin, st);
  launch_sf_velocity_update(d, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return rc;
}

int32_t pyomgpu_solve_streamfunction_begin(pyomgpu_ctx* c, pyomgpu_state* s, double* forc, pyomgpu_stream stream) {
  if (!c || !s || !forc) return fail(PYOMGPU_EINVAL, "null argument");
  if (!state_ok(s)) return fail(PYOMGPU_EINVAL, "state arrays must be device pointers with valid time levels");
  if (!is_device_ptr(forc)) return fail(PYOMGPU_EINVAL, "forc must be a device pointer");
  if (!c->have_islands) return fail(PYOMGPU_ESTATE, "islands not set up (streamfunction_init)");
  cudaStream_t st = (cudaStream_t)stream;
  StepDev d = step_dev(c, s);
  const size_t n2 = c->n2;
  launch_hydrostatic(d, st);                   // solve_streamfct.f90:24-37
  launch_sf_forcing(d, c->fpx, c->fpy, forc, st);  // :39-53 (fpx, fpy stay in the context)
  double* dp1 = s->dpsi + (size_t)(s->taup1 - 1) * n2;
  launch_first_guess(c->g, dp1, s->dpsi + (size_t)(s->tau - 1) * n2, s->dpsi + (size_t)(s->taum1 - 1) * n2, st);
  CK(cudaGetLastError());
  return PYOMGPU_OK;
}

int32_t pyomgpu_solve_streamfunction_end(pyomgpu_ctx* c, pyomgpu_state* s, pyomgpu_stream stream) {
  if (!c || !s) return fail(PYOMGPU_EINVAL, "null argument");
  if (!state_ok(s)) return fail(PYOMGPU_EINVAL, "state arrays must be device pointers with valid time levels");
  const int nisle = c->isl.nisle;
  if (nisle > 1 && (!c->have_psin || !c->have_line_psin)) return fail(PYOMGPU_ESTATE, "psin / line_psin missing");
  if (nisle > 1 && !is_device_ptr(s->dpsin)) return fail(PYOMGPU_EINVAL, "dpsin must be a device pointer");
  cudaStream_t st = (cudaStream_t)stream;
  StepDev d = step_dev(c, s);
  const size_t n2 = c->n2;
  double* dp1 = s->dpsi + (size_t)(s->taup1 - 1) * n2;
  launch_setcyclic_user(c->g, dp1, st);  // border_exchg/setcyclic (:58-59)
  if (nisle > 1) {
    if (c->lu_singular) return fail(PYOMGPU_SINGULAR, "in solve_streamfunction, lapack info not zero");
    LineGeo lg = line_geo(c);
    launch_line_integral_uv(c->nx, c->idev, lg, c->fpx, c->fpy, 1, nisle - 1, c->line_forc, st);
    launch_line_integral_psi(c->nx, c->ny, c->idev, lg, dp1, n2, 1, 1, nisle - 1, c->line_psi0, st);
    launch_island_solve(nisle, c->lu, c->ipiv, c->line_forc, c->line_psi0, s->dpsin, s->tau, st);
  }
  launch_sf_psi_update(d, c->psin, nisle, s->dpsin, st);
  launch_sf_velocity_update(d, st);
  CK(cudaGetLastError());
  return PYOMGPU_OK;
}

int32_t pyomgpu_solve_pressure(pyomgpu_ctx* c, pyomgpu_state* s, pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!c || !s) return fail(PYOMGPU_EINVAL, "null argument");
  if (!c->have_sp) return fail(PYOMGPU_ESTATE, "context has no surface-pressure operator");
  if (!state_ok(s)) return fail(PYOMGPU_EINVAL, "state arrays must be device pointers with valid time levels");
  cudaStream_t st = (cudaStream_t)stream;
  StepDev d = step_dev(c, s);
  const size_t n2 = c->n2;
  launch_hydrostatic(d, st);
  launch_sp_forcing(d, c->free_surface, c->fpx, c->fpy, c->forc, st);
  double* ps1 = s->psi + (size_t)(s->taup1 - 1) * n2;
  launch_first_guess(c->g, ps1, s->psi + (size_t)(s->tau - 1) * n2, s->psi + (size_t)(s->taum1 - 1) * n2, st);
  launch_pack(c->g, ps1, c->sol, false, st);
  pyomgpu_solve_info tmp{};
  pyomgpu_solve_info* I = info ? info : &tmp;
  int rc = run_cg_ref(c, true, c->forc, s->congr_epsilon, s->congr_max_iterations, 0.0, I, st);
  if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
  s->congr_itts = I->iterations;
  launch_unpack(c->g, c->sol, ps1, true, false, false, st);  // border_exchg/setcyclic (:71-72)
  launch_sp_velocity_update(d, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return rc;
}

}  // extern "C"
