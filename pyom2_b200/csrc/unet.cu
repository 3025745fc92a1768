// U-Net forward/backward/Adam on the tcgen05 convolution (unet.cuh).
//
// Forward and backward-data convolutions run on the tensor cores
// (conv_tc.cu; the backward-data pass is the same kernel with the flipped
// weight packing and the ReLU derivative fused as its gate).  The weight
// gradient is a CUDA-core reduction over pixels (k_conv_dw), and the
// pooling / upsampling adjoints are elementwise kernels.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "conv_tc.cuh"
#include "unet.cuh"

namespace pyomgpu {

const UNetLayer kUNet[kUNetLayers] = {
    {16, 16, 0, kEpiPlain},  // c0  X0 -> A1
    {16, 16, 0, kEpiPlain},  // c1  A1 -> S1 (+ pool P1)
    {16, 32, 1, kEpiPlain},  // c2  P1 -> A2
    {32, 32, 1, kEpiPlain},  // c3  A2 -> S2 (+ pool P2)
    {32, 64, 2, kEpiPlain},  // c4  P2 -> A3
    {64, 64, 2, kEpiPlain},  // c5  A3 -> S3 (+ pool P3)
    {64, 64, 3, kEpiPlain},  // c6  P3 -> A4
    {64, 64, 3, kEpiPlain},  // c7  A4 -> B4
    {64, 64, 3, kEpiUp},     // c8  B4 -> U3 (+ S3)
    {64, 32, 2, kEpiUp},     // c9  U3 -> U2 (+ S2)
    {32, 16, 1, kEpiUp},     // c10 U2 -> U1 (+ S1)
    {16, 16, 0, kEpiF32},    // c11 U1 -> z (channel 0)
};

size_t unet_weight_offset(int layer) {
  size_t o = 0;
  for (int l = 0; l < layer; l++) o += (size_t)9 * kUNet[l].cin * kUNet[l].cout;
  return o;
}
size_t unet_bias_offset(int layer) {
  size_t o = unet_weight_offset(kUNetLayers);
  for (int l = 0; l < layer; l++) o += (size_t)kUNet[l].cout;
  return o;
}
size_t unet_num_params() { return unet_bias_offset(kUNetLayers); }

namespace {

__device__ __forceinline__ float bfv(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ uint16_t tobf(float f) {
  __nv_bfloat16 h = __float2bfloat16_rn(f);
  return *reinterpret_cast<uint16_t*>(&h);
}

// ---------------------------------------------------------------- elementwise
// gO = planar 16-channel bf16 with channel 0 = gz, channels 1..15 = 0
__global__ void k_gz_planar(const float* __restrict__ gz, size_t npix, uint16_t* __restrict__ gO) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
    uint4 a = make_uint4((uint32_t)tobf(gz[p]), 0u, 0u, 0u);
    reinterpret_cast<uint4*>(gO)[p] = a;
    reinterpret_cast<uint4*>(gO)[npix + p] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// coarse (C, h, w) = sum over the 2x2 fine blocks of (C, 2h, 2w)
__global__ void k_up_bwd(const uint16_t* __restrict__ fine, int C, int h, int w, uint16_t* __restrict__ coarse) {
  const size_t n = (size_t)(C / 8) * h * w;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t g = e / ((size_t)h * w), rem = e - g * h * w;
    const int y = (int)(rem / w), x = (int)(rem - (size_t)y * w);
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = 0; q < 4; q++) {
      const size_t f = ((g * (2 * h) + 2 * y + (q >> 1)) * (2 * w) + 2 * x + (q & 1));
      const uint4 v = reinterpret_cast<const uint4*>(fine)[f];
      const uint32_t u[4] = {v.x, v.y, v.z, v.w};
      for (int k = 0; k < 4; k++) {
        s[2 * k] += __uint_as_float(u[k] << 16);
        s[2 * k + 1] += __uint_as_float(u[k] & 0xffff0000u);
      }
    }
    uint4 o;
    o.x = (uint32_t)tobf(s[0]) | ((uint32_t)tobf(s[1]) << 16);
    o.y = (uint32_t)tobf(s[2]) | ((uint32_t)tobf(s[3]) << 16);
    o.z = (uint32_t)tobf(s[4]) | ((uint32_t)tobf(s[5]) << 16);
    o.w = (uint32_t)tobf(s[6]) | ((uint32_t)tobf(s[7]) << 16);
    reinterpret_cast<uint4*>(coarse)[e] = o;
  }
}

// out (C, H, W) = (gdec + 0.25 gpool[y/2][x/2]) * (S > 0): the adjoint of
// "S feeds both the decoder skip and the 2x2 average pool", through S's ReLU
__global__ void k_pool_bwd_gate(const uint16_t* __restrict__ gdec, const uint16_t* __restrict__ gpool,
                                const uint16_t* __restrict__ S, int C, int H, int W, uint16_t* __restrict__ out) {
  const size_t n = (size_t)(C / 8) * H * W;
  const int h = H / 2, w = W / 2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t g = e / ((size_t)H * W), rem = e - g * H * W;
    const int y = (int)(rem / W), x = (int)(rem - (size_t)y * W);
    const uint4 a = reinterpret_cast<const uint4*>(gdec)[e];
    const uint4 b = reinterpret_cast<const uint4*>(gpool)[(g * h + y / 2) * w + x / 2];
    const uint4 s = reinterpret_cast<const uint4*>(S)[e];
    const uint32_t ua[4] = {a.x, a.y, a.z, a.w}, ub[4] = {b.x, b.y, b.z, b.w}, us[4] = {s.x, s.y, s.z, s.w};
    uint32_t o[4];
    for (int k = 0; k < 4; k++) {
      const float lo = (__uint_as_float(us[k] << 16) > 0.f)
                           ? __uint_as_float(ua[k] << 16) + 0.25f * __uint_as_float(ub[k] << 16)
                           : 0.f;
      const float hi = (__uint_as_float(us[k] & 0xffff0000u) > 0.f)
                           ? __uint_as_float(ua[k] & 0xffff0000u) + 0.25f * __uint_as_float(ub[k] & 0xffff0000u)
                           : 0.f;
      o[k] = (uint32_t)tobf(lo) | ((uint32_t)tobf(hi) << 16);
    }
    reinterpret_cast<uint4*>(out)[e] = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// ---------------------------------------------------------------- weight gradient
// dW[co][ci][tap] += sum_p G[co][p] X[ci][p + tap - (1,1)], db[co] += sum_p G[co][p].
// A CTA owns 16 output channels (blockIdx.y) and walks pixel tiles of 4 x 32;
// thread (co_l, slot) accumulates the (ci, tap) pairs slot, slot+16, ...
constexpr int kDwRows = 4, kDwCols = 32, kDwThreads = 256;

template <int CIN, int COUT>
__global__ void __launch_bounds__(kDwThreads) k_conv_dw(const uint16_t* __restrict__ X, const uint16_t* __restrict__ G,
                                                        int H, int Wd, float* __restrict__ dW, float* __restrict__ db) {
  constexpr int NACC = CIN * 9 / 16;
  constexpr int SR = kDwRows + 2, SC = kDwCols + 2;
  __shared__ uint16_t sx[CIN * SR * SC];
  __shared__ float sg[16 * kDwRows * kDwCols];
  const int tid = threadIdx.x, co_l = tid >> 4, slot = tid & 15;
  const int co = blockIdx.y * 16 + co_l;
  int off[NACC];
  float acc[NACC];
#pragma unroll
  for (int k = 0; k < NACC; k++) {
    const int q = slot + 16 * k, ci = q / 9, tap = q - 9 * ci;
    off[k] = ci * SR * SC + (tap / 3) * SC + (tap % 3);
    acc[k] = 0.f;
  }
  float accb = 0.f;
  const int tiles_x = (Wd + kDwCols - 1) / kDwCols, tiles_y = (H + kDwRows - 1) / kDwRows;
  const int ntiles = tiles_x * tiles_y;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int y0 = (t / tiles_x) * kDwRows, x0 = (t % tiles_x) * kDwCols;
    __syncthreads();
    for (int e = tid; e < CIN * SR * SC; e += kDwThreads) {
      const int ci = e / (SR * SC), rem = e - ci * SR * SC, r = rem / SC, c = rem - r * SC;
      const int y = y0 - 1 + r, x = x0 - 1 + c;
      uint16_t v = 0;
      if (y >= 0 && y < H && x >= 0 && x < Wd) v = X[(((size_t)(ci >> 3) * H + y) * Wd + x) * 8 + (ci & 7)];
      sx[e] = v;
    }
    for (int e = tid; e < 16 * kDwRows * kDwCols; e += kDwThreads) {
      const int c16 = e / (kDwRows * kDwCols), rem = e - c16 * kDwRows * kDwCols;
      const int r = rem / kDwCols, c = rem - r * kDwCols;
      const int y = y0 + r, x = x0 + c, cc = blockIdx.y * 16 + c16;
      float v = 0.f;
      if (y < H && x < Wd) v = bfv(G[(((size_t)(cc >> 3) * H + y) * Wd + x) * 8 + (cc & 7)]);
      sg[e] = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < kDwRows * kDwCols; p++) {
      const int r = p / kDwCols, c = p - r * kDwCols;
      const float g = sg[co_l * kDwRows * kDwCols + p];
      const int base = r * SC + c;
      accb += g;
#pragma unroll
      for (int k = 0; k < NACC; k++) acc[k] += g * bfv(sx[off[k] + base]);
    }
  }
#pragma unroll
  for (int k = 0; k < NACC; k++) {
    const int q = slot + 16 * k, ci = q / 9, tap = q - 9 * ci;
    atomicAdd(&dW[((size_t)co * CIN + ci) * 9 + tap], acc[k]);
  }
  if (slot == 0) atomicAdd(&db[co], accb);
}

template <int CIN, int COUT>
void launch_dw_t(const uint16_t* X, const uint16_t* G, int H, int W, float* dW, float* db, int nsm, cudaStream_t st) {
  const int ntiles = ((W + kDwCols - 1) / kDwCols) * ((H + kDwRows - 1) / kDwRows);
  const int gx = std::max(1, std::min(ntiles, 2 * nsm));
  k_conv_dw<CIN, COUT><<<dim3(gx, COUT / 16), kDwThreads, 0, st>>>(X, G, H, W, dW, db);
}

void launch_dw(int cin, int cout, const uint16_t* X, const uint16_t* G, int H, int W, float* dW, float* db, int nsm,
               cudaStream_t st) {
#define PYOMGPU_DW_CASE(a, b) \
  if (cin == a && cout == b) return launch_dw_t<a, b>(X, G, H, W, dW, db, nsm, st);
  PYOMGPU_DW_CASE(16, 16)
  PYOMGPU_DW_CASE(16, 32)
  PYOMGPU_DW_CASE(32, 32)
  PYOMGPU_DW_CASE(32, 64)
  PYOMGPU_DW_CASE(64, 64)
  PYOMGPU_DW_CASE(64, 32)
  PYOMGPU_DW_CASE(32, 16)
#undef PYOMGPU_DW_CASE
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
  }
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

int unet_alloc(UNet& n, int H, int W, bool training) {
  if (H < 8 || W < 8 || H % 8 || W % 8) return -1;
  n.H = H;
  n.W = W;
  n.training = training;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n.nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t np = unet_num_params();
  auto px = [&](int l) { return (size_t)(H >> l) * (size_t)(W >> l); };
  auto alloc = [&](void** p, size_t bytes) { return cudaMalloc(p, std::max<size_t>(bytes, 16)) == cudaSuccess; };
  bool ok = alloc((void**)&n.params, np * 4) && alloc((void**)&n.err, 16);
  for (int l = 0; l < kUNetLayers && ok; l++) {
    ok = alloc((void**)&n.wpack[l], (size_t)18 * kUNet[l].cin * kUNet[l].cout);
    if (ok && training) ok = alloc((void**)&n.wflip[l], (size_t)18 * kUNet[l].cin * kUNet[l].cout);
  }
  struct B {
    uint16_t** p;
    int c, l;
  };
  const B acts[] = {{&n.X0, 16, 0}, {&n.A1, 16, 0}, {&n.S1, 16, 0}, {&n.U1, 16, 0}, {&n.P1, 16, 1},
                    {&n.A2, 32, 1}, {&n.S2, 32, 1}, {&n.U2, 32, 1}, {&n.P2, 32, 2}, {&n.A3, 64, 2},
                    {&n.S3, 64, 2}, {&n.U3, 64, 2}, {&n.P3, 64, 3}, {&n.A4, 64, 3}, {&n.B4, 64, 3}};
  for (const B& b : acts)
    if (ok) ok = alloc((void**)b.p, 2 * (size_t)b.c * px(b.l));
  if (ok) ok = alloc((void**)&n.z, 4 * px(0));
  if (ok && training) {
    ok = alloc((void**)&n.grads, np * 4) && alloc((void**)&n.adam_m, np * 4) && alloc((void**)&n.adam_v, np * 4);
    const B grads[] = {{&n.gO, 16, 0},  {&n.gU1, 16, 0}, {&n.gv10, 16, 1}, {&n.gU2, 32, 1}, {&n.gv9, 32, 2},
                       {&n.gU3, 64, 2}, {&n.gv8, 64, 3}, {&n.gB4, 64, 3},  {&n.gA4, 64, 3}, {&n.gP3, 64, 3},
                       {&n.gS3, 64, 2}, {&n.gA3, 64, 2}, {&n.gP2, 32, 2},  {&n.gS2, 32, 1}, {&n.gA2, 32, 1},
                       {&n.gP1, 16, 1}, {&n.gS1, 16, 0}, {&n.gA1, 16, 0}};
    for (const B& b : grads)
      if (ok) ok = alloc((void**)b.p, 2 * (size_t)b.c * px(b.l));
    if (ok) ok = cudaMemset(n.adam_m, 0, np * 4) == cudaSuccess && cudaMemset(n.adam_v, 0, np * 4) == cudaSuccess;
  }
  if (ok) ok = cudaMemset(n.X0, 0, 2 * 16 * px(0)) == cudaSuccess && cudaMemset(n.params, 0, np * 4) == cudaSuccess;
  if (!ok) {
    unet_free(n);
    return -3;
  }
  return 0;
}

void unet_free(UNet& n) {
  void* ps[] = {n.params, n.grads, n.adam_m, n.adam_v, n.X0,  n.A1,  n.S1,  n.U1,   n.P1,  n.A2,  n.S2,  n.U2,
                n.P2,     n.A3,    n.S3,     n.U3,     n.P3,  n.A4,  n.B4,  n.z,    n.gO,  n.gU1, n.gv10, n.gU2,
                n.gv9,    n.gU3,   n.gv8,    n.gB4,    n.gA4, n.gP3, n.gS3, n.gA3,  n.gP2, n.gS2, n.gA2, n.gP1,
                n.gS1,    n.gA1,   n.err};
  for (void* p : ps)
    if (p) cudaFree(p);
  for (int l = 0; l < kUNetLayers; l++) {
    if (n.wpack[l]) cudaFree(n.wpack[l]);
    if (n.wflip[l]) cudaFree(n.wflip[l]);
  }
  n = UNet{};
}

void unet_pack(UNet& n, cudaStream_t st) {
  for (int l = 0; l < kUNetLayers; l++) {
    const float* w = n.params + unet_weight_offset(l);
    launch_pack_weights(w, kUNet[l].cout, kUNet[l].cin, false, n.wpack[l], st);
    if (n.training) launch_pack_weights(w, kUNet[l].cout, kUNet[l].cin, true, n.wflip[l], st);
  }
}

namespace {
int conv(UNet& n, int l, const uint16_t* x, void* y, const uint16_t* addend, uint16_t* pool, cudaStream_t st) {
  ConvSpec s{};
  s.cin = kUNet[l].cin;
  s.cout = kUNet[l].cout;
  s.H = n.H >> kUNet[l].level;
  s.W = n.W >> kUNet[l].level;
  s.x = x;
  s.wpack = n.wpack[l];
  s.bias = n.params + unet_bias_offset(l);
  s.y = y;
  s.addend = addend;
  s.pool_out = pool;
  s.relu = kUNet[l].epi != kEpiF32;
  s.epi = kUNet[l].epi;
  s.err = n.err;
  s.timeout_ns = n.timeout_ns;
  return conv3x3_launch(s, n.nsm, st);
}
// backward-data of layer l: input g (cout_l channels), output (cin_l channels), gate
int conv_bwd(UNet& n, int l, const uint16_t* g, uint16_t* y, const uint16_t* gate, cudaStream_t st) {
  ConvSpec s{};
  s.cin = kUNet[l].cout;
  s.cout = kUNet[l].cin;
  s.H = n.H >> kUNet[l].level;
  s.W = n.W >> kUNet[l].level;
  s.x = g;
  s.wpack = n.wflip[l];
  s.y = y;
  s.gate = gate;
  s.relu = 0;
  s.epi = kEpiPlain;
  s.err = n.err;
  s.timeout_ns = n.timeout_ns;
  return conv3x3_launch(s, n.nsm, st);
}
void dw(UNet& n, int l, const uint16_t* x, const uint16_t* g, cudaStream_t st) {
  launch_dw(kUNet[l].cin, kUNet[l].cout, x, g, n.H >> kUNet[l].level, n.W >> kUNet[l].level,
            n.grads + unet_weight_offset(l), n.grads + unet_bias_offset(l), n.nsm, st);
}
void up_bwd(UNet& n, const uint16_t* fine, int C, int coarse_level, uint16_t* coarse, cudaStream_t st) {
  const int h = n.H >> coarse_level, w = n.W >> coarse_level;
  const size_t m = (size_t)(C / 8) * h * w;
  k_up_bwd<<<grid_for(m), 256, 0, st>>>(fine, C, h, w, coarse);
}
void pool_bwd(UNet& n, const uint16_t* gdec, const uint16_t* gpool, const uint16_t* S, int C, int level, uint16_t* out,
              cudaStream_t st) {
  const int H = n.H >> level, W = n.W >> level;
  const size_t m = (size_t)(C / 8) * H * W;
  k_pool_bwd_gate<<<grid_for(m), 256, 0, st>>>(gdec, gpool, S, C, H, W, out);
}
}  // namespace

int unet_forward(UNet& n, cudaStream_t st) {
  int rc = 0;
  if ((rc = conv(n, 0, n.X0, n.A1, nullptr, nullptr, st))) return rc;
  if ((rc = conv(n, 1, n.A1, n.S1, nullptr, n.P1, st))) return rc;
  if ((rc = conv(n, 2, n.P1, n.A2, nullptr, nullptr, st))) return rc;
  if ((rc = conv(n, 3, n.A2, n.S2, nullptr, n.P2, st))) return rc;
  if ((rc = conv(n, 4, n.P2, n.A3, nullptr, nullptr, st))) return rc;
  if ((rc = conv(n, 5, n.A3, n.S3, nullptr, n.P3, st))) return rc;
  if ((rc = conv(n, 6, n.P3, n.A4, nullptr, nullptr, st))) return rc;
  if ((rc = conv(n, 7, n.A4, n.B4, nullptr, nullptr, st))) return rc;
  if ((rc = conv(n, 8, n.B4, n.U3, n.S3, nullptr, st))) return rc;
  if ((rc = conv(n, 9, n.U3, n.U2, n.S2, nullptr, st))) return rc;
  if ((rc = conv(n, 10, n.U2, n.U1, n.S1, nullptr, st))) return rc;
  return conv(n, 11, n.U1, n.z, nullptr, nullptr, st);
}

int unet_backward(UNet& n, const float* gz, cudaStream_t st) {
  if (!n.training) return -1;
  int rc = 0;
  const size_t np = unet_num_params();
  if (cudaMemsetAsync(n.grads, 0, np * 4, st) != cudaSuccess) return -2;
  const size_t p0 = (size_t)n.H * n.W;
  k_gz_planar<<<grid_for(p0), 256, 0, st>>>(gz, p0, n.gO);
  // output layer and decoder
  dw(n, 11, n.U1, n.gO, st);
  if ((rc = conv_bwd(n, 11, n.gO, n.gU1, n.U1, st))) return rc;
  up_bwd(n, n.gU1, 16, 1, n.gv10, st);
  dw(n, 10, n.U2, n.gv10, st);
  if ((rc = conv_bwd(n, 10, n.gv10, n.gU2, n.U2, st))) return rc;
  up_bwd(n, n.gU2, 32, 2, n.gv9, st);
  dw(n, 9, n.U3, n.gv9, st);
  if ((rc = conv_bwd(n, 9, n.gv9, n.gU3, n.U3, st))) return rc;
  up_bwd(n, n.gU3, 64, 3, n.gv8, st);
  dw(n, 8, n.B4, n.gv8, st);
  if ((rc = conv_bwd(n, 8, n.gv8, n.gB4, n.B4, st))) return rc;
  // bottom level
  dw(n, 7, n.A4, n.gB4, st);
  if ((rc = conv_bwd(n, 7, n.gB4, n.gA4, n.A4, st))) return rc;
  dw(n, 6, n.P3, n.gA4, st);
  if ((rc = conv_bwd(n, 6, n.gA4, n.gP3, nullptr, st))) return rc;
  // encoder, level 3 .. 1: S feeds the pool and the decoder skip
  pool_bwd(n, n.gU3, n.gP3, n.S3, 64, 2, n.gS3, st);
  dw(n, 5, n.A3, n.gS3, st);
  if ((rc = conv_bwd(n, 5, n.gS3, n.gA3, n.A3, st))) return rc;
  dw(n, 4, n.P2, n.gA3, st);
  if ((rc = conv_bwd(n, 4, n.gA3, n.gP2, nullptr, st))) return rc;
  pool_bwd(n, n.gU2, n.gP2, n.S2, 32, 1, n.gS2, st);
  dw(n, 3, n.A2, n.gS2, st);
  if ((rc = conv_bwd(n, 3, n.gS2, n.gA2, n.A2, st))) return rc;
  dw(n, 2, n.P1, n.gA2, st);
  if ((rc = conv_bwd(n, 2, n.gA2, n.gP1, nullptr, st))) return rc;
  pool_bwd(n, n.gU1, n.gP1, n.S1, 16, 0, n.gS1, st);
  dw(n, 1, n.A1, n.gS1, st);
  if ((rc = conv_bwd(n, 1, n.gS1, n.gA1, n.A1, st))) return rc;
  dw(n, 0, n.X0, n.gA1, st);
  return (int)cudaGetLastError();
}

void unet_adam(UNet& n, float lr, cudaStream_t st) {
  n.adam_t += 1;
  const float c1 = 1.f / (1.f - powf(0.9f, (float)n.adam_t));
  const float c2 = 1.f / (1.f - powf(0.999f, (float)n.adam_t));
  const size_t np = unet_num_params();
  k_adam<<<grid_for(np), 256, 0, st>>>(n.params, n.grads, n.adam_m, n.adam_v, np, lr, c1, c2);
  unet_pack(n, st);
}

}  // namespace pyomgpu
