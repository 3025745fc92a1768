// tcgen05 implicit-GEMM 3x3 convolution (declarations in conv_tc.cuh).
//
// One CTA of 4 warps owns a tile of kConvRows output rows x 128 output
// pixels.  Per tile: one TMA load brings the (kConvRows+2) x 130 x Cin input
// box (zero-filled outside the image = the convolution's zero padding) into
// shared memory; thread 0 issues 9 taps x Cin/16 MMAs of M=128, N=Cout, K=16
// per output row, each A operand being the box shifted by the tap offset;
// the accumulators (kConvRows x Cout f32 columns) live in TMEM and are read
// back by the 4 warps (one TMEM lane quarter each) for the fused epilogue.
// The packed weights are loaded once per CTA with a bulk copy.  Waits on
// the mbarriers are bounded by %globaltimer; on time-out the kernel records
// PYOMGPU_TIMEOUT, waits (bounded) for what it issued, frees TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>

#include "../../include/pyomgpu.h"
#include "common.cuh"
#include "conv_tc.cuh"
#include "tc.cuh"
#include "tma.cuh"

namespace pyomgpu {

namespace {

constexpr int kBW = kConvTileX + 2;  // box columns
constexpr int kBH = kConvRows + 2;   // box rows

__host__ __device__ constexpr uint32_t pow2_cols(uint32_t n) {
  uint32_t c = 32;
  while (c < n) c <<= 1;
  return c;
}

template <int CIN, int COUT>
struct ConvShape {
  static constexpr int GIN = CIN / 8;
  static constexpr uint32_t XBYTES = (uint32_t)GIN * kBH * kBW * 16;
  static constexpr uint32_t WBYTES = 9u * CIN * COUT * 2;
  static constexpr uint32_t WOFF = (XBYTES + 1023u) / 1024u * 1024u;
  static constexpr uint32_t BOFF = WOFF + (WBYTES + 127u) / 128u * 128u;
  static constexpr uint32_t MOFF = BOFF + COUT * 4;
  static constexpr uint32_t SMEM = MOFF + 64 + 1024;  // + mbarriers/TMEM address + alignment slack
  static constexpr uint32_t NCOLS = pow2_cols(kConvRows * COUT);
};

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) {
  __nv_bfloat16 h = __float2bfloat16_rn(f);
  return *reinterpret_cast<uint16_t*>(&h);
}
__device__ __forceinline__ uint32_t pack2(float a, float b) { return (uint32_t)f2bf(a) | ((uint32_t)f2bf(b) << 16); }

__device__ __forceinline__ void unpack8(const uint4& q, float (&f)[8]) {
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    f[2 * k] = __uint_as_float(w[k] << 16);
    f[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
  }
}

// Bounded mbarrier wait agreed by the whole CTA.
__device__ __forceinline__ bool cta_wait(uint64_t* bar, uint32_t parity, unsigned long long timeout_ns) {
  return __syncthreads_and(mbar_wait_bounded(bar, parity, timeout_ns)) != 0;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3x3_tc_kernel(const __grid_constant__ ConvArgs a) {
  using S = ConvShape<CIN, COUT>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sx = base;
  uint8_t* sw = base + S::WOFF;
  float* sbias = reinterpret_cast<float*>(base + S::BOFF);
  uint64_t* bar_ld = reinterpret_cast<uint64_t*>(base + S::MOFF);
  uint64_t* bar_mma = bar_ld + 1;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bar_ld + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    tc::tmem_alloc(s_tmem, S::NCOLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar_ld, 1);
    mbar_init(bar_mma, 1);
    fence_mbar_init();
  }
  for (int c = tid; c < COUT; c += kConvThreads) sbias[c] = a.bias ? a.bias[c] : 0.f;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *s_tmem;
  uint32_t ph_ld = 0, ph_mma = 0;
  bool ok = true;

  if (tid == 0) {
    mbar_arrive_expect_tx(bar_ld, S::WBYTES);
    tc::bulk_g2s(sw, a.wpack, S::WBYTES, bar_ld);
  }
  ok = cta_wait(bar_ld, ph_ld, a.timeout_ns);
  if (ok) ph_ld ^= 1u;  // on failure the phase stays the one still awaited

  const uint32_t sx_addr = smem_u32(sx), sw_addr = smem_u32(sw);
  constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, COUT);
  constexpr uint32_t kPlane = (uint32_t)kBH * kBW * 16;  // bytes between channel groups of the box

  for (int tile = blockIdx.x; ok && tile < a.ntiles; tile += gridDim.x) {
    const int ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
    const int y0 = ty * kConvRows, x0 = tx * kConvTileX;
    if (tid == 0) {
      mbar_arrive_expect_tx(bar_ld, S::XBYTES);
      tma_load_4d(sx, &a.map_x, 0, x0 - 1, y0 - 1, 0, bar_ld);
    }
    if (!cta_wait(bar_ld, ph_ld, a.timeout_ns)) {
      ok = false;
      break;
    }
    ph_ld ^= 1u;
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int t = 0; t < kConvRows; t++) {
        uint32_t acc = 0;
#pragma unroll 1
        for (int tap = 0; tap < 9; tap++) {
          const int dy = tap / 3, dx = tap - 3 * (tap / 3);
#pragma unroll
          for (int k = 0; k < CIN / 16; k++) {
            const uint32_t aaddr = sx_addr + (uint32_t)(2 * k) * kPlane + (uint32_t)((t + dy) * kBW + dx) * 16u;
            const uint32_t baddr = sw_addr + (uint32_t)((tap * S::GIN + 2 * k) * COUT) * 16u;
            const uint64_t ad = tc::smem_desc(aaddr, kPlane, 128);
            const uint64_t bd = tc::smem_desc(baddr, COUT * 16, 128);
            tc::mma_bf16(tmem + (uint32_t)(t * COUT), ad, bd, kIdesc, acc);
            acc = 1;
          }
        }
      }
      tc::commit(bar_mma);
    }
    if (!cta_wait(bar_mma, ph_mma, a.timeout_ns)) {
      ok = false;
      break;
    }
    ph_mma ^= 1u;
    tc::fence_after_sync();

    // ---- epilogue: thread = TMEM lane = output pixel x0 + 32*warp + lane
    const int m = 32 * warp + lane;
    const int x = x0 + m;
    const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll 1
    for (int t = 0; t < kConvRows; t += 2) {
#pragma unroll 1
      for (int c0 = 0; c0 < COUT; c0 += 16) {
        float v0[16], v1[16];
        tc::ld16(trow + (uint32_t)(t * COUT + c0), v0);
        tc::ld16(trow + (uint32_t)((t + 1) * COUT + c0), v1);
        tc::wait_ld();
        const int ya = y0 + t, yb = ya + 1;
        const bool in_x = x < a.W;
        if (a.epi == kEpiF32) {
          if (c0 == 0 && in_x) {
            float* y32 = reinterpret_cast<float*>(a.y);
            if (ya < a.H) y32[(size_t)ya * a.W + x] = v0[0] + sbias[0];
            if (yb < a.H) y32[(size_t)yb * a.W + x] = v1[0] + sbias[0];
          }
          continue;
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {  // two groups of 8 channels
          const int g = (c0 >> 3) + h;
          float r0[8], r1[8];
#pragma unroll
          for (int k = 0; k < 8; k++) {
            r0[k] = v0[8 * h + k] + sbias[c0 + 8 * h + k];
            r1[k] = v1[8 * h + k] + sbias[c0 + 8 * h + k];
          }
          if (a.epi == kEpiPlain) {
            float p[8];
#pragma unroll
            for (int k = 0; k < 8; k++) p[k] = 0.f;
#pragma unroll
            for (int rr = 0; rr < 2; rr++) {
              float* r = rr ? r1 : r0;
              const int yy = rr ? yb : ya;
              const bool in = in_x && yy < a.H;
              const size_t off = (((size_t)g * a.H + yy) * a.W + x) * 8;
              if (a.addend && in) {
                float q[8];
                unpack8(*reinterpret_cast<const uint4*>(a.addend + off), q);
#pragma unroll
                for (int k = 0; k < 8; k++) r[k] += q[k];
              }
              if (a.relu) {
#pragma unroll
                for (int k = 0; k < 8; k++) r[k] = fmaxf(r[k], 0.f);
              }
              if (a.gate && in) {
                float q[8];
                unpack8(*reinterpret_cast<const uint4*>(a.gate + off), q);
#pragma unroll
                for (int k = 0; k < 8; k++) r[k] = q[k] > 0.f ? r[k] : 0.f;
              }
              if (in) {
                uint4 o;
                o.x = pack2(r[0], r[1]);
                o.y = pack2(r[2], r[3]);
                o.z = pack2(r[4], r[5]);
                o.w = pack2(r[6], r[7]);
                *reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(a.y) + off) = o;
              }
#pragma unroll
              for (int k = 0; k < 8; k++) p[k] += bf2f(f2bf(r[k]));  // pool what was stored
            }
            if (a.pool_out) {  // 2x2 average: rows ya, yb in this thread, columns x, x^1 in lanes m, m^1
#pragma unroll
              for (int k = 0; k < 8; k++) p[k] += __shfl_xor_sync(0xffffffffu, p[k], 1);
              if ((lane & 1) == 0 && in_x && ya < a.H) {
                const int H2 = a.H >> 1, W2 = a.W >> 1;
                uint4 o;
                o.x = pack2(0.25f * p[0], 0.25f * p[1]);
                o.y = pack2(0.25f * p[2], 0.25f * p[3]);
                o.z = pack2(0.25f * p[4], 0.25f * p[5]);
                o.w = pack2(0.25f * p[6], 0.25f * p[7]);
                *reinterpret_cast<uint4*>(a.pool_out + (((size_t)g * H2 + (ya >> 1)) * W2 + (x >> 1)) * 8) = o;
              }
            }
          } else {  // kEpiUp: every coarse pixel feeds its 2x2 fine block
            const int H2 = 2 * a.H, W2 = 2 * a.W;
#pragma unroll
            for (int rr = 0; rr < 2; rr++) {
              const float* r = rr ? r1 : r0;
              const int yy = rr ? yb : ya;
              if (!(in_x && yy < a.H)) continue;
#pragma unroll
              for (int q4 = 0; q4 < 4; q4++) {
                const int fy = 2 * yy + (q4 >> 1), fx = 2 * x + (q4 & 1);
                const size_t off = (((size_t)g * H2 + fy) * W2 + fx) * 8;
                float s[8];
                unpack8(*reinterpret_cast<const uint4*>(a.addend + off), s);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                  s[k] += r[k];
                  if (a.relu) s[k] = fmaxf(s[k], 0.f);
                }
                uint4 o;
                o.x = pack2(s[0], s[1]);
                o.y = pack2(s[2], s[3]);
                o.z = pack2(s[4], s[5]);
                o.w = pack2(s[6], s[7]);
                *reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(a.y) + off) = o;
              }
            }
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
  }

  if (!ok) {
    if (tid == 0) atomicExch(a.err, PYOMGPU_TIMEOUT);
    // let whatever was issued land before the shared memory and TMEM go away
    mbar_wait_bounded(bar_ld, ph_ld, a.timeout_ns);
    mbar_wait_bounded(bar_mma, ph_mma, a.timeout_ns);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::NCOLS);
}

// ---------------------------------------------------------------- weights
__global__ void k_pack_weights(const float* __restrict__ w, int cout, int cin, int flip, uint16_t* __restrict__ out) {
  // forward: out[tap][ci/8][co][ci%8] = w[co][ci][tap]
  // flip:    out[tap][co/8][ci][co%8] = w[co][ci][8-tap]   (input channels = forward cout)
  const int n = 9 * cin * cout;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int co = e / (cin * 9), rem = e - co * cin * 9, ci = rem / 9, tap = rem - ci * 9;
    const float v = w[e];
    size_t o;
    if (!flip)
      o = (((size_t)tap * (cin / 8) + ci / 8) * cout + co) * 8 + (ci & 7);
    else
      o = (((size_t)(8 - tap) * (cout / 8) + co / 8) * cin + ci) * 8 + (co & 7);
    out[o] = f2bf(v);
  }
}

template <int CIN, int COUT>
int launch_one(const ConvSpec& s, int nsm, cudaStream_t st) {
  using S = ConvShape<CIN, COUT>;
  // Shared memory requested so that no more CTAs fit on an SM than its 512
  // TMEM columns hold (an allocation beyond them would wait for a CTA to exit).
  constexpr uint32_t kTmemCtas = 512u / S::NCOLS;
  constexpr uint32_t kSmemReq = std::max<uint32_t>(S::SMEM, 233472u / (kTmemCtas + 1) + 1);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSmemReq);
    if (e != cudaSuccess) return (int)e;
    attr = true;
  }
  ConvArgs a{};
  const uint64_t dims[4] = {8, (uint64_t)s.W, (uint64_t)s.H, (uint64_t)(CIN / 8)};
  const uint64_t strides[3] = {16, (uint64_t)s.W * 16, (uint64_t)s.W * s.H * 16};
  const uint32_t box[4] = {8, (uint32_t)kBW, (uint32_t)kBH, (uint32_t)(CIN / 8)};
  if (encode_map(&a.map_x, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, s.x, dims, strides, box)) return -2;
  a.wpack = s.wpack;
  a.bias = s.bias;
  a.y = s.y;
  a.gate = s.gate;
  a.addend = s.addend;
  a.pool_out = s.pool_out;
  a.H = s.H;
  a.W = s.W;
  a.tiles_x = (s.W + kConvTileX - 1) / kConvTileX;
  a.ntiles = a.tiles_x * ((s.H + kConvRows - 1) / kConvRows);
  a.relu = s.relu;
  a.epi = s.epi;
  a.err = s.err;
  a.timeout_ns = s.timeout_ns;
  // resident CTAs per SM bounded by shared memory and by TMEM columns (512 per SM)
  int per_sm = (int)std::min<uint32_t>(233472u / kSmemReq, kTmemCtas);
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(a.ntiles, per_sm * nsm));
  conv3x3_tc_kernel<CIN, COUT><<<grid, kConvThreads, kSmemReq, st>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace

bool conv3x3_supported(int cin, int cout) {
  const bool c1 = cin == 16 || cin == 32 || cin == 64;
  const bool c2 = cout == 16 || cout == 32 || cout == 64;
  return c1 && c2;
}

int conv3x3_launch(const ConvSpec& s, int nsm, cudaStream_t st) {
  if (!conv3x3_supported(s.cin, s.cout) || s.H < 1 || s.W < 1) return -1;
  if ((s.epi == kEpiUp && !s.addend) || (s.pool_out && (s.H % 2 || s.W % 2))) return -1;
#define PYOMGPU_CONV_CASE(ci, co) \
  if (s.cin == ci && s.cout == co) return launch_one<ci, co>(s, nsm, st);
  PYOMGPU_CONV_CASE(16, 16)
  PYOMGPU_CONV_CASE(16, 32)
  PYOMGPU_CONV_CASE(16, 64)
  PYOMGPU_CONV_CASE(32, 16)
  PYOMGPU_CONV_CASE(32, 32)
  PYOMGPU_CONV_CASE(32, 64)
  PYOMGPU_CONV_CASE(64, 16)
  PYOMGPU_CONV_CASE(64, 32)
  PYOMGPU_CONV_CASE(64, 64)
#undef PYOMGPU_CONV_CASE
  return -1;
}

void launch_pack_weights(const float* w, int cout, int cin, bool flip, uint16_t* wpack, cudaStream_t st) {
  const int n = 9 * cin * cout;
  k_pack_weights<<<(n + 255) / 256, 256, 0, st>>>(w, cout, cin, flip ? 1 : 0, wpack);
}

}  // namespace pyomgpu
