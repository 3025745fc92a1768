// tcgen05 implicit-GEMM 3x3 convolution (declarations in conv_tc.cuh).
//
// One CTA (8 warps) walks output tiles of ROWS rows x 128 pixels.  Per tile
// one TMA load brings the (ROWS+2) x 130 x Cin input box (zero-filled outside
// the image = the convolution's zero padding) into shared memory; thread 0
// issues 9 taps x Cin/16 MMAs of M=128, N=Cout, K=16 per output row, each A
// operand being the box shifted by the tap offset; the accumulators
// (ROWS x Cout f32 columns) live in TMEM.  The 8 warps read them back for
// the fused epilogue: warp w owns TMEM lane quarter w % 4 (32 output
// pixels) and channel half w / 4.
//
// Schedule: the packed weights (one bulk copy) and the first input box are
// requested together; input boxes are double-buffered, so the load of the
// next tile runs under the MMAs and the epilogue of the current one.  ROWS is
// 4, or 2 when Cin = 64 (two 64-channel boxes and the weights then still fit
// in shared memory, and small coarse-level images get more CTAs).
//
// Waits on the mbarriers are bounded by %globaltimer; on time-out the kernel
// records PYOMGPU_TIMEOUT, waits (bounded) for the copies and MMAs it issued,
// frees TMEM and returns.
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

__host__ __device__ constexpr uint32_t pow2_cols(uint32_t n) {
  uint32_t c = 32;
  while (c < n) c <<= 1;
  return c;
}

template <int CIN, int COUT>
struct ConvShape {
  static constexpr int ROWS = CIN == 64 ? 2 : 4;
  static constexpr int BH = ROWS + 2;
  static constexpr int GIN = CIN / 8;
  static constexpr uint32_t XBYTES = (uint32_t)GIN * BH * kBW * 16;
  static constexpr uint32_t XSTRIDE = (XBYTES + 1023u) / 1024u * 1024u;  // two buffers
  static constexpr uint32_t WBYTES = 9u * CIN * COUT * 2;
  static constexpr uint32_t WOFF = 2 * XSTRIDE;
  static constexpr uint32_t BOFF = WOFF + (WBYTES + 127u) / 128u * 128u;
  static constexpr uint32_t MOFF = BOFF + COUT * 4;
  static constexpr uint32_t SMEM = MOFF + 64 + 1024;  // + mbarriers/TMEM address + alignment slack
  static constexpr uint32_t NCOLS = pow2_cols(ROWS * COUT);
  static constexpr int CW = COUT / 2;  // channels per warpgroup
};

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) {
  __nv_bfloat16 h = __float2bfloat16_rn(f);
  return *reinterpret_cast<uint16_t*>(&h);
}
__device__ __forceinline__ uint32_t pack2(float a, float b) { return (uint32_t)f2bf(a) | ((uint32_t)f2bf(b) << 16); }
__device__ __forceinline__ uint4 pack8(const float* r) {
  uint4 o;
  o.x = pack2(r[0], r[1]);
  o.y = pack2(r[2], r[3]);
  o.z = pack2(r[4], r[5]);
  o.w = pack2(r[6], r[7]);
  return o;
}

__device__ __forceinline__ void unpack8(const uint4& q, float (&f)[8]) {
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    f[2 * k] = __uint_as_float(w[k] << 16);
    f[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
  }
}

// 8 consecutive f32 TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = __uint_as_float(r[k]);
}

// Bounded mbarrier wait agreed by the whole CTA.
__device__ __forceinline__ bool cta_wait(uint64_t* bar, uint32_t parity, unsigned long long timeout_ns) {
  return __syncthreads_and(mbar_wait_bounded(bar, parity, timeout_ns)) != 0;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3x3_tc_kernel(const __grid_constant__ ConvArgs a) {
  using S = ConvShape<CIN, COUT>;
  constexpr int ROWS = S::ROWS;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sw = base + S::WOFF;
  float* sbias = reinterpret_cast<float*>(base + S::BOFF);
  uint64_t* bar_w = reinterpret_cast<uint64_t*>(base + S::MOFF);
  uint64_t* bar_ld = bar_w + 1;  // [2], one per input buffer
  uint64_t* bar_mma = bar_w + 3;
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bar_w + 4);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, half = warp >> 2;
  if (warp == 0) {
    tc::tmem_alloc(s_tmem, S::NCOLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar_w, 1);
    mbar_init(&bar_ld[0], 1);
    mbar_init(&bar_ld[1], 1);
    mbar_init(bar_mma, 1);
    fence_mbar_init();
  }
  for (int c = tid; c < COUT; c += kConvThreads) sbias[c] = a.bias ? a.bias[c] : 0.f;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *s_tmem;
  uint32_t ph_ld[2] = {0, 0}, ph_mma = 0, ph_w = 0;
  bool ok = true;
  bool w_pending = true;
  int pend_buf = -1;  // input buffer with a load in flight that nobody waited for

  auto issue_tile = [&](int tile, int b) {
    const int ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
    mbar_arrive_expect_tx(&bar_ld[b], S::XBYTES);
    tma_load_4d(base + b * S::XSTRIDE, &a.map_x, 0, tx * kConvTileX - 1, ty * ROWS - 1, 0, &bar_ld[b]);
  };
  if (tid == 0) {
    mbar_arrive_expect_tx(bar_w, S::WBYTES);
    tc::bulk_g2s(sw, a.wpack, S::WBYTES, bar_w);
    if ((int)blockIdx.x < a.ntiles) issue_tile(blockIdx.x, 0);
  }
  if ((int)blockIdx.x < a.ntiles) pend_buf = 0;
  ok = cta_wait(bar_w, ph_w, a.timeout_ns);
  if (ok) {
    ph_w ^= 1u;
    w_pending = false;
  }

  const uint32_t sw_addr = smem_u32(sw);
  constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, COUT);
  constexpr uint32_t kPlane = (uint32_t)S::BH * kBW * 16;  // bytes between channel groups of the box

  int it = 0;
  for (int tile = blockIdx.x; ok && tile < a.ntiles; tile += gridDim.x, ++it) {
    const int b = it & 1;
    const int ty = tile / a.tiles_x, tx = tile - ty * a.tiles_x;
    const int y0 = ty * ROWS, x0 = tx * kConvTileX;
    if (!cta_wait(&bar_ld[b], ph_ld[b], a.timeout_ns)) {
      ok = false;
      break;
    }
    ph_ld[b] ^= 1u;
    pend_buf = -1;
    const int next = tile + gridDim.x;
    if (tid == 0) {
      // buffer b^1 was read by the MMAs of the previous tile, which completed
      if (next < a.ntiles) issue_tile(next, b ^ 1);
      tc::fence_after_sync();
      const uint32_t sx_addr = smem_u32(base + b * S::XSTRIDE);
#pragma unroll 1
      for (int t = 0; t < ROWS; t++) {
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
    if (next < a.ntiles) pend_buf = b ^ 1;
    if (!cta_wait(bar_mma, ph_mma, a.timeout_ns)) {
      ok = false;
      break;
    }
    ph_mma ^= 1u;
    tc::fence_after_sync();

    // ---- epilogue: lane = output pixel x0 + 32*quarter + lane, channels [half*CW, (half+1)*CW)
    const int x = x0 + 32 * quarter + lane;
    const bool in_x = x < a.W;
    const uint32_t trow = tmem + ((uint32_t)(32 * quarter) << 16);
#pragma unroll 1
    for (int t = 0; t < ROWS; t += 2) {
      const int ya = y0 + t, yb = ya + 1;
#pragma unroll 1
      for (int c0 = half * S::CW; c0 < (half + 1) * S::CW; c0 += 8) {
        float r0[8], r1[8];
        tmem_ld8(trow + (uint32_t)(t * COUT + c0), r0);
        tmem_ld8(trow + (uint32_t)((t + 1) * COUT + c0), r1);
        tc::wait_ld();
#pragma unroll
        for (int k = 0; k < 8; k++) {
          r0[k] += sbias[c0 + k];
          r1[k] += sbias[c0 + k];
        }
        if (a.epi == kEpiF32) {
          if (c0 == 0 && in_x) {
            float* y32 = reinterpret_cast<float*>(a.y);
            if (ya < a.H) y32[(size_t)ya * a.W + x] = r0[0];
            if (yb < a.H) y32[(size_t)yb * a.W + x] = r1[0];
          }
          continue;
        }
        const int g = c0 >> 3;
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
            if (in) *reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(a.y) + off) = pack8(r);
#pragma unroll
            for (int k = 0; k < 8; k++) p[k] += bf2f(f2bf(r[k]));  // pool what was stored
          }
          if (a.pool_out) {  // 2x2 average: rows ya, yb in this thread, columns x, x^1 in lanes l, l^1
#pragma unroll
            for (int k = 0; k < 8; k++) p[k] = 0.25f * (p[k] + __shfl_xor_sync(0xffffffffu, p[k], 1));
            if ((lane & 1) == 0 && in_x && ya < a.H) {
              const int H2 = a.H >> 1, W2 = a.W >> 1;
              *reinterpret_cast<uint4*>(a.pool_out + (((size_t)g * H2 + (ya >> 1)) * W2 + (x >> 1)) * 8) = pack8(p);
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
            for (int fy = 0; fy < 2; fy++) {
              const size_t off = (((size_t)g * H2 + 2 * yy + fy) * W2 + 2 * x) * 8;
              uint4 s2[2];
              s2[0] = *reinterpret_cast<const uint4*>(a.addend + off);
              s2[1] = *reinterpret_cast<const uint4*>(a.addend + off + 8);
              uint4 o2[2];
#pragma unroll
              for (int fx = 0; fx < 2; fx++) {
                float s[8];
                unpack8(s2[fx], s);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                  s[k] += r[k];
                  if (a.relu) s[k] = fmaxf(s[k], 0.f);
                }
                o2[fx] = pack8(s);
              }
              uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(a.y) + off);
              dst[0] = o2[0];
              dst[1] = o2[1];
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
    if (w_pending) mbar_wait_bounded(bar_w, ph_w, a.timeout_ns);
    if (pend_buf >= 0) mbar_wait_bounded(&bar_ld[pend_buf], ph_ld[pend_buf], a.timeout_ns);
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
  static_assert(kSmemReq <= 232448u, "shared memory of one CTA");
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
  const uint32_t box[4] = {8, (uint32_t)kBW, (uint32_t)S::BH, (uint32_t)(CIN / 8)};
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
  a.ntiles = a.tiles_x * ((s.H + S::ROWS - 1) / S::ROWS);
  a.relu = s.relu;
  a.epi = s.epi;
  a.err = s.err;
  a.timeout_ns = s.timeout_ns;
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
