// Learned preconditioner (U-Net of unet.cuh) and the flexible CG that uses
// it -- the C ABI's pyomgpu_precond_* and pyomgpu_solve_fcg.  No counterpart
// in the reference, whose only preconditioner is Jacobi
// (make_inv_sfc, solve_streamfct.f90:381-422).
//
// Network input (16 planar bf16 channels, 4 used) on the image of the
// interior points, pixel (x, y) = Fortran (x+1, y+1), padded with zeros to
// multiples of 8: the residual scaled to unit rms over the unknowns, the
// unknown mask (Z != 0), hur / mean(hur) and cosu.  Its output, masked, is a
// search direction approximating the error A^-1 r in the units
// e * dbar / rms(r), dbar = mean |diag A| over the unknowns.
//
// Training loss (one residual/error pair): the relative energy-norm error
// ||z - e^||_S^2 / ||e^||_S^2 of the network output z against the scaled
// error e^ = (x* - x) dbar / rms(r), with ||u||_S^2 = -u^T D A u,
// D = dxu dyu cosu (A = D^-1 S, S symmetric negative definite).
//
// Solver: flexible CG over two directions per iteration, the Jacobi
// direction Z r and the network direction N(r) (Bridson and Greif's
// multi-preconditioned CG, truncated to the previous block): the block W is
// A-orthogonalised against the previous block P in the D inner product
// (which makes A self-adjoint), then x moves by the energy-optimal
// combination of the two new directions.  Every iteration is therefore at
// least a Jacobi-preconditioned step, and the network only has to supply the
// smooth error Jacobi cannot remove.  FP64 vectors and dot products; the
// iteration is captured once into a CUDA graph and replayed.  A stall hands
// the iterate to the Jacobi-PCG kernel; the FP64 true residual decides.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cg_ref.cuh"
#include "ctx.h"
#include "kernels.cuh"
#include "unet.cuh"

using namespace pyomgpu;

namespace pyomgpu {
void set_last_error(const char* msg);
}

struct pyomgpu_precond {
  pyomgpu_ctx* c = nullptr;
  UNet net;
  int Hp = 0, Wp = 0;
  float4* stat = nullptr;  // per pixel: mask, hur/mean, cosu, 0
  double nu = 0;           // number of unknowns
  double dbar = 1;         // mean |diag A| over the unknowns
  // solver vectors (padded FP64)
  double *r = nullptr, *w1 = nullptr, *w2 = nullptr, *aw1 = nullptr, *aw2 = nullptr;
  double *p1 = nullptr, *p2 = nullptr, *ap1 = nullptr, *ap2 = nullptr, *t1 = nullptr, *t2 = nullptr;
  double* part = nullptr;  // per-block partials
  double* sc = nullptr;    // device scalars
  double* h_sc = nullptr;  // pinned copy
  float* gz = nullptr;     // [Hp][Wp]
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t graph_stream = nullptr;
};

namespace {

constexpr int kRB = 256;       // threads of the vector kernels
constexpr int kRBlocks = 592;  // blocks of the reducing vector kernels (4 x 148)
constexpr int kMaxNV = 5;      // partials per block

// device scalar slots
enum : int {
  kRR = 0, kBB, kRtol2BB, kDone, kIters, kMaxIt, kBreak,
  kT11, kT12, kT21, kT22,          // <A p_i, w_j>_D
  kB11, kB12, kB21, kB22,          // orthogonalisation coefficients
  kG11, kG12, kG22, kRank,         // Gram matrix <p_i, A p_j>_D of the previous block, its rank
  kC1, kC2,                        // step coefficients
  kLoss, kK1, kK2, kFirst,
  kNSc = 32
};

int pfail(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

__device__ __forceinline__ double dweight(const double* dxu, const double* dyu, const double* cosu, int i, int j) {
  return dxu[i + 1] * dyu[j + 1] * cosu[j + 1];
}

// Block partial sums of NV values, written to part[blockIdx.x * NV + k].
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* part) {
  __shared__ double sh[kRB / 32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double x = v[k];
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) x += __shfl_xor_sync(0xffffffffu, x, m);
    if (lane == 0) sh[w][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int q = 0; q < kRB / 32; q++) s += sh[q][threadIdx.x];
    part[blockIdx.x * NV + threadIdx.x] = s;
  }
}

// Sum of the partials of nv values (fixed order) into out[0..nv), by one warp.
__device__ __forceinline__ void sum_partials(const double* __restrict__ part, int nb, int nv, double* out) {
  double v[kMaxNV] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += 32)
    for (int k = 0; k < nv; k++) v[k] += part[b * nv + k];
  for (int k = 0; k < nv; k++) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], m);
    out[k] = v[k];
  }
}

__global__ void k_set_scalar(double* sc, int idx, double v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc[idx] = v;
}

// ---------------------------------------------------------------- image <-> field
__global__ void k_static(Geo g, const double* __restrict__ W, const double* __restrict__ hur,
                         const double* __restrict__ cosu, double hur_scale, int Hp, int Wp, float4* __restrict__ stat) {
  const size_t n = (size_t)Hp * Wp;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(e / Wp), x = (int)(e - (size_t)y * Wp);
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    if (x < g.nx && y < g.ny) {
      const int i = x + 1, j = y + 1;
      const bool m = W[g.at(i, j)] != 0.0;
      s.x = m ? 1.f : 0.f;
      s.y = m ? (float)(hur[fidx(g.nx, i, j)] * hur_scale) : 0.f;
      s.z = (float)cosu[j + 1];
    }
    stat[e] = s;
  }
}

__device__ __forceinline__ uint16_t f2bf_rn(float f) {
  uint32_t u = __float_as_uint(f);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// X0 group 0 = (r / rms(r) masked, mask, hur, cos, 0, 0, 0, 0)
__global__ void k_prep(Geo g, const double* __restrict__ r, const double* __restrict__ sc, double nu,
                       const float4* __restrict__ stat, int Hp, int Wp, uint16_t* __restrict__ X0) {
  if (sc[kDone] != 0.0) return;
  const double rr = sc[kRR];
  const double inv = rr > 0.0 ? 1.0 / sqrt(rr / nu) : 0.0;
  const size_t n = (size_t)Hp * Wp;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(e / Wp), x = (int)(e - (size_t)y * Wp);
    const float4 s = stat[e];
    float rv = 0.f;
    if (x < g.nx && y < g.ny && s.x != 0.f) rv = (float)(r[g.at(x + 1, y + 1)] * inv);
    uint4 o;
    o.x = (uint32_t)f2bf_rn(rv) | ((uint32_t)f2bf_rn(s.x) << 16);
    o.y = (uint32_t)f2bf_rn(s.y) | ((uint32_t)f2bf_rn(s.z) << 16);
    o.z = 0u;
    o.w = 0u;
    reinterpret_cast<uint4*>(X0)[e] = o;
  }
}

// w1 = Z r (Jacobi direction), w2 = mask * network output (cyclic copies)
__global__ void k_dirs(Geo g, const float* __restrict__ zn, const float4* __restrict__ stat, int Wp,
                       const double* __restrict__ Z, const double* __restrict__ r, const double* __restrict__ sc,
                       double* __restrict__ w1, double* __restrict__ w2) {
  if (sc[kDone] != 0.0) return;
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(e / g.nx), x = (int)(e - (size_t)y * g.nx);
    const size_t pi = (size_t)y * Wp + x, k = g.at(x + 1, y + 1);
    store_cyclic(w1, g, x + 1, y + 1, Z[k] * r[k]);
    store_cyclic(w2, g, x + 1, y + 1, stat[pi].x != 0.f ? (double)zn[pi] : 0.0);
  }
}

// aw = A w for both directions; partials <A p_i, w_j>_D (previous block)
__global__ void k_apply_w(Geo g, OpDev<double> op, const double* __restrict__ w1, const double* __restrict__ w2,
                          const double* __restrict__ ap1, const double* __restrict__ ap2, const double* dxu,
                          const double* dyu, const double* cosu, const double* __restrict__ sc,
                          double* __restrict__ aw1, double* __restrict__ aw2, double* __restrict__ part) {
  double v[4] = {0, 0, 0, 0};
  if (sc[kDone] == 0.0) {
    const size_t n = (size_t)g.nx * g.ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
      const int j = (int)(e / g.nx) + 1, i = (int)(e - (size_t)(j - 1) * g.nx) + 1;
      const size_t k = g.at(i, j);
      aw1[k] = apply_point(op, g, w1, i, j);
      aw2[k] = apply_point(op, g, w2, i, j);
      const double d = dweight(dxu, dyu, cosu, i, j);
      const double a1 = d * ap1[k], a2 = d * ap2[k];
      v[0] += a1 * w1[k];
      v[1] += a1 * w2[k];
      v[2] += a2 * w1[k];
      v[3] += a2 * w2[k];
    }
  }
  block_partials<4>(v, part);
}

// P_new = W - P B, AP_new = AW - AP B (in place); partials <p1,ap1>, <p1,ap2>, <p2,ap2>, <p1,r>, <p2,r> (D)
__global__ void k_new_block(Geo g, const double* __restrict__ w1, const double* __restrict__ w2,
                            const double* __restrict__ aw1, const double* __restrict__ aw2,
                            const double* __restrict__ r, const double* dxu, const double* dyu, const double* cosu,
                            const double* __restrict__ sc, double* __restrict__ p1, double* __restrict__ p2,
                            double* __restrict__ ap1, double* __restrict__ ap2, double* __restrict__ part) {
  double v[5] = {0, 0, 0, 0, 0};
  if (sc[kDone] == 0.0) {
    const double b11 = sc[kB11], b12 = sc[kB12], b21 = sc[kB21], b22 = sc[kB22];
    const size_t n = (size_t)g.nx * g.ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
      const int j = (int)(e / g.nx) + 1, i = (int)(e - (size_t)(j - 1) * g.nx) + 1;
      const size_t k = g.at(i, j);
      const double po1 = p1[k], po2 = p2[k], qo1 = ap1[k], qo2 = ap2[k];
      const double n1 = w1[k] - (po1 * b11 + po2 * b21), n2 = w2[k] - (po1 * b12 + po2 * b22);
      const double m1 = aw1[k] - (qo1 * b11 + qo2 * b21), m2 = aw2[k] - (qo1 * b12 + qo2 * b22);
      store_cyclic(p1, g, i, j, n1);
      store_cyclic(p2, g, i, j, n2);
      ap1[k] = m1;
      ap2[k] = m2;
      const double d = dweight(dxu, dyu, cosu, i, j);
      v[0] += d * n1 * m1;
      v[1] += d * n1 * m2;
      v[2] += d * n2 * m2;
      v[3] += d * n1 * r[k];
      v[4] += d * n2 * r[k];
    }
  }
  block_partials<5>(v, part);
}

// x += c1 p1 + c2 p2, r -= c1 ap1 + c2 ap2 (unknowns); partial sum r^2
__global__ void k_step(Geo g, const double* __restrict__ W, const double* __restrict__ p1,
                       const double* __restrict__ p2, const double* __restrict__ ap1, const double* __restrict__ ap2,
                       const double* __restrict__ sc, double* __restrict__ x, double* __restrict__ r,
                       double* __restrict__ part) {
  double v[1] = {0.0};
  if (sc[kDone] == 0.0) {
    const double c1 = sc[kC1], c2 = sc[kC2];
    const size_t n = (size_t)g.nx * g.ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
      const int j = (int)(e / g.nx) + 1, i = (int)(e - (size_t)(j - 1) * g.nx) + 1;
      const size_t k = g.at(i, j);
      if (W[k] == 0.0) continue;
      x[k] += c1 * p1[k] + c2 * p2[k];
      const double rv = r[k] - (c1 * ap1[k] + c2 * ap2[k]);
      store_cyclic(r, g, i, j, rv);
      v[0] += rv * rv;
    }
  }
  block_partials<1>(v, part);
}

// r = mask (forc - A x); partials sum r^2, sum forc^2 over the unknowns
__global__ void k_residual_vec(Geo g, OpDev<double> op, const double* __restrict__ forc, const double* __restrict__ x,
                               double* __restrict__ r, double* __restrict__ part) {
  double v[2] = {0.0, 0.0};
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / g.nx) + 1, i = (int)(e - (size_t)(j - 1) * g.nx) + 1;
    const bool m = op.W[g.at(i, j)] != 0.0;
    const double f = forc[fidx(g.nx, i, j)];
    const double rv = m ? f - apply_point(op, g, x, i, j) : 0.0;
    store_cyclic(r, g, i, j, rv);
    if (m) {
      v[0] += rv * rv;
      v[1] += f * f;
    }
  }
  block_partials<2>(v, part);
}

// r_pad = mask * r_user (cyclic copies); partial sum r^2 over the unknowns
__global__ void k_mask_rr(Geo g, const double* __restrict__ W, const double* __restrict__ r_user,
                          double* __restrict__ r, double* __restrict__ part) {
  double v[1] = {0.0};
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / g.nx) + 1, i = (int)(e - (size_t)(j - 1) * g.nx) + 1;
    const double rv = W[g.at(i, j)] != 0.0 ? r_user[fidx(g.nx, i, j)] : 0.0;
    store_cyclic(r, g, i, j, rv);
    v[0] += rv * rv;
  }
  block_partials<1>(v, part);
}

// 2x2 symmetric solve G c = h; rank 1 (second direction dropped) when G is
// numerically singular.  Returns the rank (0 if even g11 vanishes).
__device__ int solve2(double g11, double g12, double g22, double h1, double h2, double& c1, double& c2) {
  const double det = g11 * g22 - g12 * g12;
  if (g11 != 0.0 && g22 != 0.0 && fabs(det) > 1e-10 * fabs(g11 * g22)) {
    c1 = (h1 * g22 - g12 * h2) / det;
    c2 = (g11 * h2 - g12 * h1) / det;
    return 2;
  }
  c2 = 0.0;
  if (g11 != 0.0) {
    c1 = h1 / g11;
    return 1;
  }
  c1 = 0.0;
  return 0;
}

// stage 0: initial residual; 1: T -> B; 2: G, h -> c; 3: rr -> done?; 4: rr only
__global__ void k_scalars(const double* __restrict__ part, int nb, int stage, double* __restrict__ sc) {
  const int nv = stage == 0 ? 2 : stage == 1 ? 4 : stage == 2 ? 5 : 1;
  double s[kMaxNV];
  sum_partials(part, nb, nv, s);
  if (threadIdx.x != 0) return;
  if (stage == 0) {
    sc[kRR] = s[0];
    sc[kBB] = s[1];
    sc[kRtol2BB] = sc[kRtol2BB] * s[1];
    sc[kDone] = (s[0] <= sc[kRtol2BB]) ? 1.0 : 0.0;
    sc[kIters] = 0.0;
    sc[kBreak] = 0.0;
    sc[kFirst] = 1.0;
    sc[kRank] = 0.0;
    return;
  }
  if (stage == 4) {
    sc[kRR] = s[0];
    return;
  }
  if (sc[kDone] != 0.0) return;
  if (stage == 1) {
    // B = Gprev^-1 T (columns j = 1, 2); zero for the first block
    double b11 = 0, b12 = 0, b21 = 0, b22 = 0;
    if (sc[kFirst] == 0.0) {
      const int rank = (int)sc[kRank];
      const double g11 = sc[kG11], g12 = sc[kG12], g22 = sc[kG22];
      if (rank == 2) {
        solve2(g11, g12, g22, s[0], s[2], b11, b21);
        solve2(g11, g12, g22, s[1], s[3], b12, b22);
      } else if (rank == 1) {
        b11 = s[0] / g11;
        b12 = s[1] / g11;
      }
    }
    sc[kT11] = s[0];
    sc[kT12] = s[1];
    sc[kT21] = s[2];
    sc[kT22] = s[3];
    sc[kB11] = b11;
    sc[kB12] = b12;
    sc[kB21] = b21;
    sc[kB22] = b22;
  } else if (stage == 2) {
    double c1 = 0, c2 = 0;
    const int rank = solve2(s[0], s[1], s[2], s[3], s[4], c1, c2);
    const bool finite = c1 == c1 && c2 == c2 && s[0] == s[0];
    if (rank == 0 || !finite) {
      sc[kBreak] = 1.0;
      sc[kDone] = 1.0;
      c1 = c2 = 0.0;
    }
    sc[kG11] = s[0];
    sc[kG12] = s[1];
    sc[kG22] = s[2];
    sc[kRank] = rank;
    sc[kC1] = c1;
    sc[kC2] = rank == 2 ? c2 : 0.0;
    sc[kFirst] = 0.0;
  } else {
    sc[kRR] = s[0];
    sc[kIters] += 1.0;
    if (!(s[0] == s[0])) {
      sc[kBreak] = 1.0;
      sc[kDone] = 1.0;
    } else if (s[0] <= sc[kRtol2BB] || sc[kIters] >= sc[kMaxIt]) {
      sc[kDone] = 1.0;
    }
  }
}

// ---------------------------------------------------------------- training loss
// Zp = mask * zn, Ep = mask * e * scale (padded FP64 with cyclic copies), scale = dbar / rms(r)
__global__ void k_loss_fields(Geo g, const float* __restrict__ zn, const double* __restrict__ e_user,
                              const float4* __restrict__ stat, int Wp, const double* __restrict__ sc, double nu,
                              double dbar, double* __restrict__ Zp, double* __restrict__ Ep) {
  const double rr = sc[kRR];
  const double scale = rr > 0.0 ? dbar / sqrt(rr / nu) : 0.0;
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(k / g.nx), x = (int)(k - (size_t)y * g.nx);
    const bool m = stat[(size_t)y * Wp + x].x != 0.f;
    store_cyclic(Zp, g, x + 1, y + 1, m ? (double)zn[(size_t)y * Wp + x] : 0.0);
    store_cyclic(Ep, g, x + 1, y + 1, m ? e_user[fidx(g.nx, x + 1, y + 1)] * scale : 0.0);
  }
}

// SZ = D A Zp, SE = D A Ep; partials a = z^T S e, b = z^T S z, c = e^T S e
__global__ void k_loss_dots(Geo g, OpDev<double> op, const double* __restrict__ Zp, const double* __restrict__ Ep,
                            const double* dxu, const double* dyu, const double* cosu, double* __restrict__ SZ,
                            double* __restrict__ SE, double* __restrict__ part) {
  double v[3] = {0.0, 0.0, 0.0};
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / g.nx) + 1, i = (int)(e - (size_t)(j - 1) * g.nx) + 1;
    const size_t k = g.at(i, j);
    const double d = dweight(dxu, dyu, cosu, i, j);
    const double sz = d * apply_point(op, g, Zp, i, j), se = d * apply_point(op, g, Ep, i, j);
    SZ[k] = sz;
    SE[k] = se;
    v[0] += Zp[k] * se;
    v[1] += Zp[k] * sz;
    v[2] += Ep[k] * se;
  }
  block_partials<3>(v, part);
}

// loss = (b - 2a + c) / c (all three are S forms, S negative definite); d loss / d z = (2/c)(S z - S e)
__global__ void k_loss_scalars(const double* __restrict__ part, int nb, double* __restrict__ sc) {
  double s[kMaxNV];
  sum_partials(part, nb, 3, s);
  if (threadIdx.x != 0) return;
  const double a = s[0], b = s[1], c = s[2];
  const bool ok = c != 0.0 && a == a && b == b && c == c;
  sc[kLoss] = ok ? (b - 2.0 * a + c) / c : 1.0;
  sc[kK1] = ok ? 2.0 / c : 0.0;
  sc[kK2] = ok ? -2.0 / c : 0.0;
}

__global__ void k_loss_grad(Geo g, const double* __restrict__ SZ, const double* __restrict__ SE,
                            const float4* __restrict__ stat, int Hp, int Wp, const double* __restrict__ sc,
                            float* __restrict__ gz) {
  const double k1 = sc[kK1], k2 = sc[kK2];
  const size_t n = (size_t)Hp * Wp;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(e / Wp), x = (int)(e - (size_t)y * Wp);
    float v = 0.f;
    if (x < g.nx && y < g.ny && stat[e].x != 0.f) {
      const size_t k = g.at(x + 1, y + 1);
      v = (float)(k1 * SZ[k] + k2 * SE[k]);
    }
    gz[e] = v;
  }
}

__global__ void k_unpad(Geo g, const double* __restrict__ a, double* __restrict__ user) {
  const size_t n = (size_t)(g.nx + 4) * (g.ny + 4);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / (g.nx + 4)) - 1, i = (int)(e - (size_t)(j + 1) * (g.nx + 4)) - 1;
    user[e] = a[g.at(i, j)];
  }
}

int blocks_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + kRB - 1) / kRB, kRBlocks)); }

bool is_dev(const void* p) {
  cudaPointerAttributes a;
  if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// P->r = mask * r_user and sc[kRR] (the network's input scaling)
void load_r(pyomgpu_precond* P, const double* r_user, cudaStream_t st) {
  const Geo& g = P->c->g;
  const int nb = blocks_for((size_t)g.nx * g.ny);
  k_mask_rr<<<nb, kRB, 0, st>>>(g, P->c->sf.W, r_user, P->r, P->part);
  k_scalars<<<1, 32, 0, st>>>(P->part, nb, 4, P->sc);
  k_set_scalar<<<1, 1, 0, st>>>(P->sc, kDone, 0.0);
}

// network output for P->r (sc[kRR] must hold sum r^2 over the unknowns) -> P->net.z
int run_net(pyomgpu_precond* P, cudaStream_t st) {
  const size_t npx = (size_t)P->Hp * P->Wp;
  k_prep<<<blocks_for(npx), kRB, 0, st>>>(P->c->g, P->r, P->sc, P->nu, P->stat, P->Hp, P->Wp, P->net.X0);
  return unet_forward(P->net, st);
}

// One solver iteration (launch sequence captured into the graph).
int iteration(pyomgpu_precond* P, cudaStream_t st) {
  pyomgpu_ctx* c = P->c;
  const Geo& g = c->g;
  const int nb = blocks_for((size_t)g.nx * g.ny);
  if (int rc = run_net(P, st)) return rc;
  k_dirs<<<nb, kRB, 0, st>>>(g, P->net.z, P->stat, P->Wp, c->sf.W, P->r, P->sc, P->w1, P->w2);
  k_apply_w<<<nb, kRB, 0, st>>>(g, c->sf.dev(), P->w1, P->w2, P->ap1, P->ap2, c->dxu, c->dyu, c->cosu, P->sc, P->aw1,
                                P->aw2, P->part);
  k_scalars<<<1, 32, 0, st>>>(P->part, nb, 1, P->sc);
  k_new_block<<<nb, kRB, 0, st>>>(g, P->w1, P->w2, P->aw1, P->aw2, P->r, c->dxu, c->dyu, c->cosu, P->sc, P->p1,
                                  P->p2, P->ap1, P->ap2, P->part);
  k_scalars<<<1, 32, 0, st>>>(P->part, nb, 2, P->sc);
  k_step<<<nb, kRB, 0, st>>>(g, c->sf.W, P->p1, P->p2, P->ap1, P->ap2, P->sc, c->sol, P->r, P->part);
  k_scalars<<<1, 32, 0, st>>>(P->part, nb, 3, P->sc);
  return (int)cudaGetLastError();
}
constexpr int kLaunchesPerIteration = 1 + kUNetLayers + 7;

int ensure_graph(pyomgpu_precond* P) {
  if (P->exec) return 0;
  if (!P->graph_stream && cudaStreamCreateWithFlags(&P->graph_stream, cudaStreamNonBlocking) != cudaSuccess)
    return -2;
  cudaStream_t s = P->graph_stream;
  // one uncaptured pass first: per-kernel attributes are set on first launch
  if (int rc = unet_forward(P->net, s)) return rc;
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -2;
  int rc = iteration(P, s);
  cudaGraph_t gph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &gph);
  if (rc || e != cudaSuccess || !gph) {
    if (gph) cudaGraphDestroy(gph);
    cudaGetLastError();
    return rc ? rc : -2;
  }
  if (cudaGraphInstantiate(&P->exec, gph, 0) != cudaSuccess) {
    cudaGraphDestroy(gph);
    return -2;
  }
  P->graph = gph;
  return 0;
}

// Static input channels, unknown count and mean |diag A| of grid c (host reductions, once per grid).
int bind_grid(pyomgpu_precond* P, pyomgpu_ctx* c) {
  P->c = c;
  const size_t Pn = c->g.size(), npx = (size_t)P->Hp * P->Wp;
  std::vector<double> Wh(Pn), hur(c->n2);
  if (cudaMemcpy(Wh.data(), c->sf.W, Pn * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(hur.data(), c->hur, c->n2 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -2;
  double nu = 0, hs = 0, ds = 0;
  for (int j = 1; j <= c->ny; j++)
    for (int i = 1; i <= c->nx; i++) {
      const double z = Wh[c->g.at(i, j)];
      if (z != 0.0) {
        nu += 1;
        hs += hur[fidx(c->nx, i, j)];
        ds += 1.0 / std::fabs(z);
      }
    }
  P->nu = std::max(1.0, nu);
  P->dbar = nu > 0 ? ds / nu : 1.0;
  const double hscale = hs > 0 ? nu / hs : 1.0;
  k_static<<<blocks_for(npx), kRB>>>(c->g, c->sf.W, c->hur, c->cosu, hscale, P->Hp, P->Wp, P->stat);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
}

}  // namespace

extern "C" {

int64_t pyomgpu_precond_num_params(void) { return (int64_t)unet_num_params(); }

int32_t pyomgpu_precond_create(pyomgpu_ctx* c, int32_t training, pyomgpu_precond** out) {
  if (!c || !out) return pfail(PYOMGPU_EINVAL, "precond_create: null argument");
  *out = nullptr;
  if (!c->have_islands) return pfail(PYOMGPU_ESTATE, "precond_create: set up the islands first (Z is an input)");
  auto* P = new pyomgpu_precond();
  P->c = c;
  P->Hp = (c->ny + 7) / 8 * 8;
  P->Wp = (c->nx + 7) / 8 * 8;
  if (unet_alloc(P->net, P->Hp, P->Wp, training != 0)) {
    delete P;
    return pfail(PYOMGPU_ENOMEM, "precond_create: network buffers");
  }
  const size_t Pn = c->g.size(), npx = (size_t)P->Hp * P->Wp;
  bool ok = true;
  for (double** a : {&P->r, &P->w1, &P->w2, &P->aw1, &P->aw2, &P->p1, &P->p2, &P->ap1, &P->ap2, &P->t1, &P->t2})
    ok = ok && cudaMalloc((void**)a, Pn * sizeof(double)) == cudaSuccess &&
         cudaMemset(*a, 0, Pn * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&P->stat, npx * sizeof(float4)) == cudaSuccess &&
       cudaMalloc((void**)&P->part, (size_t)kRBlocks * kMaxNV * sizeof(double)) == cudaSuccess &&
       cudaMalloc((void**)&P->sc, kNSc * sizeof(double)) == cudaSuccess &&
       cudaMallocHost((void**)&P->h_sc, kNSc * sizeof(double)) == cudaSuccess &&
       cudaMalloc((void**)&P->gz, npx * sizeof(float)) == cudaSuccess;
  if (!ok) {
    pyomgpu_precond_destroy(P);
    return pfail(PYOMGPU_ENOMEM, "precond_create: cudaMalloc");
  }
  cudaMemset(P->sc, 0, kNSc * sizeof(double));
  if (bind_grid(P, c)) {
    pyomgpu_precond_destroy(P);
    return pfail(PYOMGPU_ECUDA, "precond_create: set-up kernels failed");
  }
  *out = P;
  return PYOMGPU_OK;
}

int32_t pyomgpu_precond_rebind(pyomgpu_precond* P, pyomgpu_ctx* c) {
  if (!P || !c) return pfail(PYOMGPU_EINVAL, "precond_rebind: null argument");
  if (c->nx != P->c->nx || c->ny != P->c->ny || c->g.pitch != P->c->g.pitch)
    return pfail(PYOMGPU_EINVAL, "precond_rebind: the grids differ in size");
  if (!c->have_islands) return pfail(PYOMGPU_ESTATE, "precond_rebind: set up the islands first (Z is an input)");
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  P->exec = nullptr;
  P->graph = nullptr;
  return bind_grid(P, c) ? pfail(PYOMGPU_ECUDA, "precond_rebind: set-up kernels failed") : PYOMGPU_OK;
}

void pyomgpu_precond_destroy(pyomgpu_precond* P) {
  if (!P) return;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  if (P->graph_stream) cudaStreamDestroy(P->graph_stream);
  unet_free(P->net);
  for (void* a : {(void*)P->r, (void*)P->w1, (void*)P->w2, (void*)P->aw1, (void*)P->aw2, (void*)P->p1, (void*)P->p2,
                  (void*)P->ap1, (void*)P->ap2, (void*)P->t1, (void*)P->t2, (void*)P->stat, (void*)P->part,
                  (void*)P->sc, (void*)P->gz})
    if (a) cudaFree(a);
  if (P->h_sc) cudaFreeHost(P->h_sc);
  delete P;
}

int32_t pyomgpu_precond_set_params(pyomgpu_precond* P, const float* params, int64_t n) {
  if (!P || !params || n != (int64_t)unet_num_params()) return pfail(PYOMGPU_EINVAL, "set_params: wrong size");
  if (cudaMemcpy(P->net.params, params, (size_t)n * 4, cudaMemcpyDefault) != cudaSuccess)
    return pfail(PYOMGPU_ECUDA, "set_params: copy");
  unet_pack(P->net, 0);
  P->net.adam_t = 0;
  if (P->net.training) {
    cudaMemset(P->net.adam_m, 0, (size_t)n * 4);
    cudaMemset(P->net.adam_v, 0, (size_t)n * 4);
  }
  return cudaDeviceSynchronize() == cudaSuccess ? PYOMGPU_OK : pfail(PYOMGPU_ECUDA, "set_params: pack");
}

int32_t pyomgpu_precond_get_params(pyomgpu_precond* P, float* params, int64_t n) {
  if (!P || !params || n != (int64_t)unet_num_params()) return pfail(PYOMGPU_EINVAL, "get_params: wrong size");
  return cudaMemcpy(params, P->net.params, (size_t)n * 4, cudaMemcpyDefault) == cudaSuccess
             ? PYOMGPU_OK
             : pfail(PYOMGPU_ECUDA, "get_params: copy");
}

int32_t pyomgpu_precond_get_grads(pyomgpu_precond* P, float* grads, int64_t n) {
  if (!P || !grads || !P->net.training || n != (int64_t)unet_num_params())
    return pfail(PYOMGPU_EINVAL, "get_grads: not a training preconditioner or wrong size");
  return cudaMemcpy(grads, P->net.grads, (size_t)n * 4, cudaMemcpyDefault) == cudaSuccess
             ? PYOMGPU_OK
             : pfail(PYOMGPU_ECUDA, "get_grads: copy");
}

int32_t pyomgpu_unet_forward_backward(pyomgpu_precond* P, const uint16_t* x0, const float* gz, float* z,
                                      pyomgpu_stream stream) {
  if (!P || !x0 || !z) return pfail(PYOMGPU_EINVAL, "unet_forward_backward: null argument");
  if (gz && !P->net.training) return pfail(PYOMGPU_EINVAL, "unet_forward_backward: not a training preconditioner");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t npx = (size_t)P->Hp * P->Wp;
  // both may be host memory: stage them in the network's own device buffers
  cudaMemcpyAsync(P->net.X0, x0, npx * 32, cudaMemcpyDefault, st);
  if (gz) cudaMemcpyAsync(P->gz, gz, npx * sizeof(float), cudaMemcpyDefault, st);
  cudaMemsetAsync(P->net.err, 0, sizeof(int), st);
  int rc = unet_forward(P->net, st);
  if (!rc && gz) rc = unet_backward(P->net, P->gz, st);
  if (rc) return pfail(PYOMGPU_ECUDA, "unet_forward_backward: launch failed");
  cudaMemcpyAsync(z, P->net.z, npx * 4, cudaMemcpyDefault, st);
  int err = 0;
  cudaMemcpyAsync(&err, P->net.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return pfail(PYOMGPU_ECUDA, "unet_forward_backward: kernel failed");
  if (err) return pfail(PYOMGPU_TIMEOUT, "unet_forward_backward: a wait ran out");
  return PYOMGPU_OK;
}

int32_t pyomgpu_precond_apply(pyomgpu_precond* P, const double* r, double* z, pyomgpu_stream stream) {
  if (!P || !r || !z) return pfail(PYOMGPU_EINVAL, "precond_apply: null argument");
  if (!is_dev(r) || !is_dev(z)) return pfail(PYOMGPU_EINVAL, "precond_apply: r and z must be device arrays");
  cudaStream_t st = (cudaStream_t)stream;
  pyomgpu_ctx* c = P->c;
  load_r(P, r, st);
  cudaMemsetAsync(P->net.err, 0, sizeof(int), st);
  if (run_net(P, st)) return pfail(PYOMGPU_ECUDA, "precond_apply: network launch failed");
  const int nb = blocks_for((size_t)c->nx * c->ny);
  k_dirs<<<nb, kRB, 0, st>>>(c->g, P->net.z, P->stat, P->Wp, c->sf.W, P->r, P->sc, P->t1, P->t2);
  k_unpad<<<blocks_for(c->n2), kRB, 0, st>>>(c->g, P->t2, z);
  int err = 0;
  cudaMemcpyAsync(&err, P->net.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return pfail(PYOMGPU_ECUDA, "precond_apply: kernel failed");
  return err ? pfail(PYOMGPU_TIMEOUT, "precond_apply: a wait ran out") : PYOMGPU_OK;
}

int32_t pyomgpu_precond_train_step(pyomgpu_precond* P, const double* r, const double* e, float lr, float* loss,
                                   pyomgpu_stream stream) {
  if (!P || !r || !e) return pfail(PYOMGPU_EINVAL, "train_step: null argument");
  if (!P->net.training) return pfail(PYOMGPU_EINVAL, "train_step: not a training preconditioner");
  if (!is_dev(r) || !is_dev(e)) return pfail(PYOMGPU_EINVAL, "train_step: r and e must be device arrays");
  cudaStream_t st = (cudaStream_t)stream;
  pyomgpu_ctx* c = P->c;
  const Geo& g = c->g;
  const int nb = blocks_for((size_t)c->nx * c->ny);
  load_r(P, r, st);
  cudaMemsetAsync(P->net.err, 0, sizeof(int), st);
  if (run_net(P, st)) return pfail(PYOMGPU_ECUDA, "train_step: forward launch failed");
  const size_t npx = (size_t)P->Hp * P->Wp;
  k_loss_fields<<<nb, kRB, 0, st>>>(g, P->net.z, e, P->stat, P->Wp, P->sc, P->nu, P->dbar, P->w1, P->w2);
  k_loss_dots<<<nb, kRB, 0, st>>>(g, c->sf.dev(), P->w1, P->w2, c->dxu, c->dyu, c->cosu, P->t1, P->t2, P->part);
  k_loss_scalars<<<1, 32, 0, st>>>(P->part, nb, P->sc);
  k_loss_grad<<<blocks_for(npx), kRB, 0, st>>>(g, P->t1, P->t2, P->stat, P->Hp, P->Wp, P->sc, P->gz);
  if (unet_backward(P->net, P->gz, st)) return pfail(PYOMGPU_ECUDA, "train_step: backward launch failed");
  if (lr > 0.f) unet_adam(P->net, lr, st);
  cudaMemcpyAsync(P->h_sc, P->sc, kNSc * sizeof(double), cudaMemcpyDeviceToHost, st);
  int err = 0;
  cudaMemcpyAsync(&err, P->net.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return pfail(PYOMGPU_ECUDA, "train_step: kernel failed");
  if (err) return pfail(PYOMGPU_TIMEOUT, "train_step: a wait ran out");
  if (loss) *loss = (float)P->h_sc[kLoss];
  return PYOMGPU_OK;
}

int32_t pyomgpu_solve_fcg(pyomgpu_ctx* c, pyomgpu_precond* P, const double* forc, double* sol, double rtol,
                          int32_t max_it, pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!c || !P || P->c != c || !forc || !sol || !(rtol > 0) || max_it < 1)
    return pfail(PYOMGPU_EINVAL, "solve_fcg: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  pyomgpu_solve_info tmp{};
  pyomgpu_solve_info* I = info ? info : &tmp;
  *I = pyomgpu_solve_info{};
  const bool f_dev = is_dev(forc), s_dev = is_dev(sol);
  const double* f = forc;
  if (!f_dev) {
    cudaMemcpyAsync(c->stage_a, forc, c->n2 * sizeof(double), cudaMemcpyHostToDevice, st);
    f = c->stage_a;
  }
  const double* s_in = sol;
  if (!s_dev) {
    cudaMemcpyAsync(c->stage_b, sol, c->n2 * sizeof(double), cudaMemcpyHostToDevice, st);
    s_in = c->stage_b;
  }
  launch_pack(c->g, s_in, c->sol, true, st);
  if (ensure_graph(P)) return pfail(PYOMGPU_ECUDA, "solve_fcg: graph capture failed");
  cudaEventRecord(c->e0, st);
  const Geo& g = c->g;
  const int nb = blocks_for((size_t)g.nx * g.ny);
  for (double* a : {P->p1, P->p2, P->ap1, P->ap2}) cudaMemsetAsync(a, 0, g.size() * sizeof(double), st);
  k_set_scalar<<<1, 1, 0, st>>>(P->sc, kRtol2BB, rtol * rtol);
  k_set_scalar<<<1, 1, 0, st>>>(P->sc, kMaxIt, (double)max_it);
  k_residual_vec<<<nb, kRB, 0, st>>>(g, c->sf.dev(), f, c->sol, P->r, P->part);
  k_scalars<<<1, 32, 0, st>>>(P->part, nb, 0, P->sc);
  cudaMemsetAsync(P->net.err, 0, sizeof(int), st);
  int launches = 5;
  // the captured iteration runs on its own stream: order it after st
  cudaEvent_t ev = nullptr;
  cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cudaEventRecord(ev, st);
  cudaStreamWaitEvent(P->graph_stream, ev, 0);
  // stall: the best residual so far has not dropped by 1 % for kStallIts
  // iterations (the residual of CG-type methods is not monotone)
  constexpr int kStallIts = 48;
  double best_rr = -1.0;
  int best_it = 0;
  const bool trace = std::getenv("PYOMGPU_FCG_TRACE") != nullptr;
  const int chunk = 4;
  for (int it = 0; it < max_it; it += chunk) {
    for (int k = 0; k < chunk; k++) cudaGraphLaunch(P->exec, P->graph_stream);
    launches += chunk * kLaunchesPerIteration;
    cudaMemcpyAsync(P->h_sc, P->sc, kNSc * sizeof(double), cudaMemcpyDeviceToHost, P->graph_stream);
    if (cudaStreamSynchronize(P->graph_stream) != cudaSuccess) {
      cudaEventDestroy(ev);
      return pfail(PYOMGPU_ECUDA, "solve_fcg: iteration failed");
    }
    const double rr_now = P->h_sc[kRR];
    const int it_now = (int)P->h_sc[kIters];
    if (trace)
      std::fprintf(stderr, "fcg it %d rel.res %.3e c %.3e %.3e rank %d\n", it_now,
                   P->h_sc[kBB] > 0 ? std::sqrt(rr_now / P->h_sc[kBB]) : std::sqrt(rr_now), P->h_sc[kC1],
                   P->h_sc[kC2], (int)P->h_sc[kRank]);
    if (P->h_sc[kDone] != 0.0) break;
    if (best_rr < 0.0 || rr_now < 0.9801 * best_rr) {
      best_rr = rr_now;
      best_it = it_now;
    } else if (it_now - best_it >= kStallIts) {
      break;
    }
  }
  cudaEventRecord(ev, P->graph_stream);
  cudaStreamWaitEvent(st, ev, 0);
  cudaEventDestroy(ev);
  int err = 0;
  cudaMemcpyAsync(&err, P->net.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (err) return pfail(PYOMGPU_TIMEOUT, "solve_fcg: a wait ran out");
  const int fcg_it = (int)P->h_sc[kIters];
  I->iterations = fcg_it;
  I->fcg_iterations = fcg_it;
  I->outer_iterations = 1;
  // the FP64 true residual decides; Jacobi-PCG takes over on a stall, a breakdown or a miss
  launch_fill_cyclic(c->g, c->sol, st);
  launch_residual(c->g, c->sf.dev(), f, c->sol, c->part, 1024, c->scal, st);
  cudaMemcpyAsync(c->h_scal, c->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  launches += 3;
  double rr = c->h_scal[0], bb = c->h_scal[1];
  int rc = PYOMGPU_OK;
  if (!(rr <= rtol * rtol * bb) && fcg_it < max_it) {
    pyomgpu_solve_info J{};
    rc = run_pcg_from_sol(c, f, max_it - fcg_it, rtol, &J, st);
    if (rc < 0 || rc == PYOMGPU_TIMEOUT) return rc;
    I->iterations += J.iterations;
    I->outer_iterations = 2;
    launches += 1;
    launch_fill_cyclic(c->g, c->sol, st);
    launch_residual(c->g, c->sf.dev(), f, c->sol, c->part, 1024, c->scal, st);
    cudaMemcpyAsync(c->h_scal, c->scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    launches += 3;
    rr = c->h_scal[0];
    bb = c->h_scal[1];
  }
  if (s_dev) {
    launch_unpack(c->g, c->sol, sol, false, false, false, st);
  } else {
    launch_unpack(c->g, c->sol, c->stage_b, false, false, false, st);
    cudaMemcpyAsync(sol, c->stage_b, c->n2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  }
  cudaEventRecord(c->e1, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return pfail(PYOMGPU_ECUDA, "solve_fcg: final copies failed");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->e0, c->e1);
  I->device_ms = ms;
  I->kernel_launches = launches + 2;
  I->rel_residual = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
  I->estimated_error = I->rel_residual;
  const bool conv = rr <= rtol * rtol * bb;
  I->converged = conv ? 1 : 0;
  I->status = conv ? PYOMGPU_OK : (rr == rr ? PYOMGPU_MAXITER : PYOMGPU_NAN);
  return I->status;
}

}  // extern "C"
