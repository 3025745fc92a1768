// C ABI of the learned preconditioner (include/pyomgpu.h, "learned
// preconditioner" section): tcgen05 convolution entry points.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/pyomgpu.h"
#include "conv_tc.cuh"

using namespace pyomgpu;

namespace pyomgpu {
void set_last_error(const char* msg);
}

namespace {

int lfail(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

bool on_device(const void* p) {
  if (!p) return true;  // optional arguments
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

}  // namespace

extern "C" {

int32_t pyomgpu_conv3x3_bf16(int32_t cin, int32_t cout, int32_t H, int32_t W, const uint16_t* x, const float* w,
                             const float* bias, int32_t relu, int32_t epilogue, const uint16_t* gate,
                             const uint16_t* addend, void* y, uint16_t* pool_out, int32_t flip,
                             pyomgpu_stream stream) {
  if (!x || !w || !y || H < 1 || W < 1) return lfail(PYOMGPU_EINVAL, "conv3x3: null pointer or empty image");
  if (!conv3x3_supported(cin, cout)) return lfail(PYOMGPU_EINVAL, "conv3x3: channel counts must be 16, 32 or 64");
  if (epilogue < kEpiPlain || epilogue > kEpiF32) return lfail(PYOMGPU_EINVAL, "conv3x3: unknown epilogue");
  for (const void* p : {(const void*)x, (const void*)w, (const void*)bias, (const void*)gate, (const void*)addend,
                        (const void*)y, (const void*)pool_out})
    if (!on_device(p)) return lfail(PYOMGPU_EINVAL, "conv3x3: every array must be in device memory");
  cudaStream_t st = (cudaStream_t)stream;
  uint16_t* wpack = nullptr;
  int* err = nullptr;
  if (cudaMalloc(&wpack, sizeof(uint16_t) * 9 * cin * cout) != cudaSuccess ||
      cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
    cudaFree(wpack);
    return lfail(PYOMGPU_ENOMEM, "conv3x3: cudaMalloc");
  }
  // flip: w is the forward weight [cin][cout][3][3] of the layer this call differentiates
  if (flip)
    launch_pack_weights(w, cin, cout, true, wpack, st);
  else
    launch_pack_weights(w, cout, cin, false, wpack, st);
  cudaMemsetAsync(err, 0, sizeof(int), st);
  ConvSpec s{};
  s.cin = cin;
  s.cout = cout;
  s.H = H;
  s.W = W;
  s.x = x;
  s.wpack = wpack;
  s.bias = bias;
  s.y = y;
  s.gate = gate;
  s.addend = addend;
  s.pool_out = pool_out;
  s.relu = relu;
  s.epi = epilogue;
  s.err = err;
  s.timeout_ns = 2000000000ull;
  int rc = conv3x3_launch(s, sm_count(), st);
  int herr = 0;
  cudaError_t e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(wpack);
  cudaFree(err);
  if (rc == -1) return lfail(PYOMGPU_EINVAL, "conv3x3: unsupported shape or epilogue arguments");
  if (rc == -2) return lfail(PYOMGPU_ECUDA, "conv3x3: tensor map encoding failed");
  if (rc != 0) return lfail(PYOMGPU_ECUDA, cudaGetErrorString((cudaError_t)rc));
  if (e != cudaSuccess) return lfail(PYOMGPU_ECUDA, cudaGetErrorString(e));
  if (herr) return lfail(PYOMGPU_TIMEOUT, "conv3x3: a wait ran out");
  return PYOMGPU_OK;
}

}  // extern "C"
