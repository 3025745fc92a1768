// Pipelined Jacobi-PCG: one TMA-staged sweep and one grid barrier per iteration.
//
// Same iterates as the reference's congrad_streamfunction (solve_streamfct.f90:
// 223-299) in exact arithmetic.  Sweep n, with alpha_{n-1} and beta_n/beta_{n-1}
// from the previous barrier, works on a tile plus a one-cell halo staged in
// shared memory (r_{n-2}, As_{n-1}, s_{n-1}, Z, FX, FY):
//
//   r_{n-1} = r_{n-2} - alpha_{n-1} As_{n-1}         (tile + halo)
//   x_{n-1} = x_{n-2} + alpha_{n-1} s_{n-1}          (own points)
//   s_n     = Z r_{n-1} + (beta_n/beta_{n-1}) s_{n-1} (tile + halo)
//   As_n    = A s_n                                    (own points)
//
// and reduces (s_n, As_n), (Z r_{n-1}, As_n), (Z As_n, As_n) and ||r_{n-1}||^2.
// After the barrier alpha_n = beta_n / (s_n, As_n) and, because Z is diagonal,
//   beta_{n+1} = (Z r_n, r_n) = beta_n - 2 alpha_n (Z r_{n-1}, As_n) + alpha_n^2 (Z As_n, As_n),
// so the second reduction of the textbook loop disappears.  r, As and s are
// double-buffered (neighbour tiles read their halos while they are rewritten).
//
// T = double: FP64 PCG.  T = float: inner solver of the mixed-precision path,
// all products accumulated in FP64.
#include <math.h>

#include "cg_pipe.cuh"

namespace pyomgpu {

namespace {
constexpr int kPX = 72;  // box columns: Fortran i0-4 .. i0+67 (16-byte aligned origin for FP32 and FP64)
constexpr int kPY = kTileY + 2;
constexpr int kPOff = 4;  // box column of Fortran i0
constexpr int kNV = 5;    // (s,As), (Zr,As), (Z As,As), ||r||^2, (Zr,r)

template <typename T>
__host__ __device__ constexpr size_t tile_bytes() {
  return ((size_t)kPX * kPY * sizeof(T) + 127) / 128 * 128;
}
}  // namespace

template <typename T>
__global__ void __launch_bounds__(kPipeThreads, 3) cg_pipe_kernel(const __grid_constant__ PipeParams<T> P) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr size_t TB = tile_bytes<T>();
  T* tr = reinterpret_cast<T*>(smem);
  T* tA = reinterpret_cast<T*>(smem + TB);
  T* ts = reinterpret_cast<T*>(smem + 2 * TB);
  T* tZ = reinterpret_cast<T*>(smem + 3 * TB);
  T* tFX = reinterpret_cast<T*>(smem + 4 * TB);
  T* tFY = reinterpret_cast<T*>(smem + 5 * TB);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 6 * TB);

  const Geo g = P.g;
  const OpDev<T> op = P.op;
  const unsigned nb = gridDim.x;
  const int ntiles = P.ntx * P.nty;
  unsigned long long epoch = 0;
  uint32_t phase = 0;

  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();

  // ---- r0 = b - A x; beta_1 = (Z r0, r0) -----------------------------------------
  {
    double v[3] = {0.0, 0.0, 0.0};
    for (int t = blockIdx.x; t < ntiles; t += nb) {
      const int i0 = 1 + kTileX * (t % P.ntx), j0 = 1 + kTileY * (t / P.ntx);
      for (int e = threadIdx.x; e < kTileX * kTileY; e += kPipeThreads) {
        const int i = i0 + e % kTileX, j = j0 + e / kTileX;
        if (i > g.nx || j > g.ny) continue;
        const size_t o = g.at(i, j);
        const T bv = P.b[o];
        const T r = bv - apply_point(op, g, P.x, i, j);
        store_cyclic(P.r[0], g, i, j, r);
        store_cyclic(P.r[1], g, i, j, r);
        const T z = op.W[o];
        v[0] += (double)z * (double)r * (double)r;
        if (z != T(0)) {
          v[1] += (double)bv * (double)bv;
          v[2] += (double)r * (double)r;
        }
      }
    }
    double out[3];
    block_reduce<3, -1, kPipeThreads>(v, out);
    if (threadIdx.x == 0) {
      double* s = P.slots + (size_t)blockIdx.x * 8;
      for (int k = 0; k < 3; k++) s[k] = out[k];
    }
  }
  if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns)) return;
  double red[kNV];
  grid_collect<3, -1, kPipeThreads>(P.slots, 8, nb, *reinterpret_cast<double(*)[3]>(red));
  double beta = red[0];
  const double bb = red[1];
  double rr = red[2];
  const double tol2 = P.rtol * P.rtol * bb;
  int it = 0, status = PYOMGPU_OK;
  double a_prev = 0.0, bq = 0.0;  // alpha_0 = 0, s_0 = 0
  if (rr <= tol2) goto done;

  for (int n = 1;; n++) {
    {
      const T a = (T)a_prev, q = (T)bq;
      const int in = n & 1, outb = (n - 1) & 1;  // r_{n-2} in r[n&1]; As_{n-1}, s_{n-1} in [(n-1)&1]
      T* __restrict__ rout = P.r[outb];
      T* __restrict__ Aout = P.A[n & 1];
      T* __restrict__ sout = P.s[n & 1];
      double v[kNV] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int t = blockIdx.x; t < ntiles; t += nb) {
        const int i0 = 1 + kTileX * (t % P.ntx), j0 = 1 + kTileY * (t / P.ntx);
        __syncthreads();  // previous tile's shared-memory reads are done
        if (threadIdx.x == 0) {
          fence_proxy_async_smem();
          fence_proxy_async_global();
          mbar_arrive_expect_tx(bar, 6u * kPX * kPY * (uint32_t)sizeof(T));
          const int ex = i0 - kPOff + 1 + kXOff, ey = j0;  // element column of Fortran i0-4, row of j0-1
          tma_load_2d(tr, &P.map_r[in], ex, ey, bar);
          tma_load_2d(tA, &P.map_A[outb], ex, ey, bar);
          tma_load_2d(ts, &P.map_s[outb], ex, ey, bar);
          tma_load_2d(tZ, &P.map_Z, ex, ey, bar);
          tma_load_2d(tFX, &P.map_FX, ex, ey, bar);
          tma_load_2d(tFY, &P.map_FY, ex, ey, bar);
        }
        const bool ok = __syncthreads_and(mbar_wait_bounded(bar, phase, P.timeout_ns));
        phase ^= 1u;
        if (!ok) {
          if (threadIdx.x == 0) atomicExch(&P.ctl->error, PYOMGPU_TIMEOUT);
          return;
        }
        // tile + one-cell halo: box columns kPOff-1 .. kPOff+kTileX, all rows
        for (int e = threadIdx.x; e < (kTileX + 2) * kPY; e += kPipeThreads) {
          const int ii = kPOff - 1 + e % (kTileX + 2), jj = e / (kTileX + 2);
          const int k = jj * kPX + ii;
          const T rn = tr[k] - a * tA[k];
          const T so = ts[k];
          const int i = i0 - kPOff + ii, j = j0 - 1 + jj;
          if (ii >= kPOff && ii < kPOff + kTileX && jj >= 1 && jj <= kTileY && i <= g.nx && j <= g.ny) {
            const size_t o = g.at(i, j);
            P.x[o] = P.x[o] + a * so;  // x_{n-1}
            store_cyclic(rout, g, i, j, rn);
          }
          tr[k] = rn;
          ts[k] = tZ[k] * rn + q * so;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kTileX * kTileY; e += kPipeThreads) {
          const int c = e % kTileX, rrw = e / kTileX;
          const int i = i0 + c, j = j0 + rrw;
          if (i > g.nx || j > g.ny) continue;
          const int k = (rrw + 1) * kPX + c + kPOff;
          const T sc = ts[k];
          const T As = op.ax[i + 1] * op.bx[j + 1] * (tFX[k + 1] * (ts[k + 1] - sc) + tFX[k] * (ts[k - 1] - sc)) +
                       op.by[j + 1] * (tFY[k + kPX] * (ts[k + kPX] - sc) + tFY[k] * (ts[k - kPX] - sc));
          store_cyclic(sout, g, i, j, sc);
          store_cyclic(Aout, g, i, j, As);
          const double z = (double)tZ[k], r1 = (double)tr[k], ad = (double)As;
          v[0] += (double)sc * ad;
          v[1] += z * r1 * ad;
          v[2] += z * ad * ad;
          v[4] += z * r1 * r1;
          if (z != 0.0) v[3] += r1 * r1;
        }
      }
      double out[kNV];
      block_reduce<kNV, -1, kPipeThreads>(v, out);
      if (threadIdx.x == 0) {
        double* s = P.slots + (size_t)((epoch & 1) * nb + blockIdx.x) * 8;
        for (int k = 0; k < kNV; k++) s[k] = out[k];
      }
    }
    const unsigned long long ep = epoch;
    if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns)) return;
    grid_collect<kNV, -1, kPipeThreads>(P.slots + (size_t)((ep & 1) * nb) * 8, 8, nb, red);
    rr = red[3];
    it = n - 1;  // x_{n-1}, r_{n-1} are current
    if (rr <= tol2) break;
    if (it >= P.max_it) {
      status = PYOMGPU_MAXITER;
      break;
    }
    // beta_n itself, reduced directly from r_{n-1}, replaces the value the
    // expansion predicted at the previous barrier, so expansion errors do not
    // accumulate from one iteration to the next
    const double beta_n = red[4];
    const double alpha = beta_n / red[0];
    const double bnext = beta_n - 2.0 * alpha * red[1] + alpha * alpha * red[2];
    if (!(alpha == alpha) || !(bnext == bnext) || !(rr == rr)) {
      status = PYOMGPU_NAN;
      break;
    }
    a_prev = alpha;
    bq = bnext / beta_n;
    beta = bnext;
  }
done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.out->iterations = it;
    P.out->status = status;
    P.out->rr = rr;
    P.out->bb = bb;
  }
}

template __global__ void cg_pipe_kernel<double>(const __grid_constant__ PipeParams<double> P);
template __global__ void cg_pipe_kernel<float>(const __grid_constant__ PipeParams<float> P);

const void* cg_pipe_kernel_ptr(bool f32) {
  return f32 ? (const void*)cg_pipe_kernel<float> : (const void*)cg_pipe_kernel<double>;
}

// tensor map with the pipelined kernel's kPX x kPY box
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_pipe_map(CUtensorMap* map, const void* base, const Geo& g, bool f32) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return -1;
    fn = (EncodeTiledFn)p;
  }
  const size_t es_bytes = f32 ? 4 : 8;
  const cuuint64_t dims[2] = {(cuuint64_t)g.pitch, (cuuint64_t)(g.ny + 2 * kOnx)};
  const cuuint64_t strides[1] = {(cuuint64_t)g.pitch * es_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)kPX, (cuuint32_t)kPY};
  const cuuint32_t es[2] = {1, 1};
  return (int)fn(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)base, dims,
                 strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

template <typename T>
int pipe_encode_all(PipeParams<T>& P) {
  const bool f32 = sizeof(T) == 4;
  for (int k = 0; k < 2; k++)
    if (encode_pipe_map(&P.map_r[k], P.r[k], P.g, f32) || encode_pipe_map(&P.map_A[k], P.A[k], P.g, f32) ||
        encode_pipe_map(&P.map_s[k], P.s[k], P.g, f32))
      return -1;
  if (encode_pipe_map(&P.map_Z, P.op.W, P.g, f32) || encode_pipe_map(&P.map_FX, P.op.FX, P.g, f32) ||
      encode_pipe_map(&P.map_FY, P.op.FY, P.g, f32))
    return -1;
  return 0;
}
template int pipe_encode_all<double>(PipeParams<double>&);
template int pipe_encode_all<float>(PipeParams<float>&);

size_t pipe_smem_bytes(bool f32) { return 6 * (f32 ? tile_bytes<float>() : tile_bytes<double>()) + 128; }

}  // namespace pyomgpu
