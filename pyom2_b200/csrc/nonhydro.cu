// Non-hydrostatic pressure solve on the GPU: congrad_non_hydro
// (non_hydrostatic.f90:146-242) as one persistent, grid-synchronised kernel,
// apply_op_3D (:247-276) as a stand-alone kernel, and their C ABI.
//
// Per CG iteration the kernel makes two sweeps over bricks of 32 x ty x kc
// cells, separated by grid barriers that carry the reductions (dot_3D /
// absmax_3D, :279-322).  A brick's operands come into shared memory by TMA
// through a two-stage pipeline (the next brick loads while this one is
// computed), and every warp marches up one column of the brick with the
// field below, at and above its cell in registers:
//
//   sweep A  boxes (brick + one-cell halo) of res and s_{n-1}; forms
//            s_n = res + bq s_{n-1} in the box; partial sums of
//            (s_n, A s_n) and max|s_n| over maskT; writes s_n
//   sweep B  the s_n box, res and p of the brick; A s_n again;
//            res -= alpha A s_n (in place), p += alpha s_n; partial
//            sums of (res, res)
//
// An iteration streams 64 bytes per cell from HBM (res and s_{n-1} read, s_n
// written and read back, res and p read and written) plus the flag byte
// twice, and stores no A s vector.  The search direction alternates between
// two buffers (s_{n-1} is still read by neighbouring bricks while s_n is
// written).  The convergence test of iteration n needs max|s_{n+1}|, so it
// runs after sweep A of iteration n+1, exactly as the reference evaluates it
// after forming the new direction.  Cyclic halos are written by the owner of
// the source cell (setcyclic_xyz); the kernel is compiled for each
// combination of cyclic x / cyclic y so that closed domains carry no halo
// logic.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "../../include/pyomgpu.h"
#include "cg_ref.cuh"
#include "nonhydro.cuh"
#include "tma.cuh"

namespace cg = cooperative_groups;

namespace pyomgpu {

void set_last_error(const char* msg);

namespace {

__device__ __forceinline__ size_t fidx3(int nx, int ny, int i, int j, int k) {
  return (size_t)(i + 1) + (size_t)(nx + 2 * kOnx) * ((size_t)(j + 1) + (size_t)(ny + 2 * kOnx) * (size_t)(k - 1));
}

// Cell of lane `lane` in work unit u: a run of 32 consecutive i on row (j,k).
__device__ __forceinline__ void nh_unit(uint32_t u, uint32_t nch, uint32_t ny, int lane, int& i, int& j, int& k) {
  const uint32_t row = u / nch;
  const uint32_t ch = u - row * nch;
  const uint32_t kk = row / ny;
  j = (int)(row - kk * ny) + 1;
  k = (int)kk + 1;
  i = (int)(ch * 32u) + lane + 1;
}

__device__ __forceinline__ ptrdiff_t nh_off(const NHGeo& G, int di, int dj, int dk) {
  return (ptrdiff_t)di + (ptrdiff_t)dj * G.g.pitch + (ptrdiff_t)dk * (ptrdiff_t)G.plane;
}

// Offsets (relative to cell (i,j) on the same level) of the setcyclic_xyz halo
// copies of (i,j); 0 = none.  At most three: x, y and the corner.
template <bool CX, bool CY>
__device__ __forceinline__ void nh_copy_offsets(const Geo& g, int i, int j, ptrdiff_t& ox, ptrdiff_t& oy) {
  ox = 0;
  oy = 0;
  if (CX) ox = (i <= kOnx) ? (ptrdiff_t)g.nx : ((i > g.nx - kOnx) ? -(ptrdiff_t)g.nx : 0);
  if (CY) oy = (j <= kOnx) ? (ptrdiff_t)g.ny * g.pitch : ((j > g.ny - kOnx) ? -(ptrdiff_t)g.ny * g.pitch : 0);
}
template <bool CX, bool CY>
__device__ __forceinline__ void nh_put(double* __restrict__ a, size_t q, ptrdiff_t ox, ptrdiff_t oy, double v) {
  a[q] = v;
  if (CX && ox) a[q + ox] = v;
  if (CY && oy) {
    a[q + oy] = v;
    if (CX && ox) a[q + ox + oy] = v;
  }
}
template <bool CX, bool CY>
__device__ __forceinline__ void nh_add_halo(double* __restrict__ a, size_t q, ptrdiff_t ox, ptrdiff_t oy, double d) {
  if (CX && ox) a[q + ox] += d;
  if (CY && oy) {
    a[q + oy] += d;
    if (CX && ox) a[q + ox + oy] += d;
  }
}

}  // namespace

// Pipeline state of a block: per stage a "full" mbarrier (the TMA copy
// landed) and an "empty" one (all eight warps are done with the stage).
struct NHPipe {
  uint64_t* full;
  uint64_t* empty;
  uint32_t fph;   // per stage: parity of the next full phase to wait for (all threads)
  uint32_t eph;   // per stage: parity of the next empty phase to wait for (thread 0)
  uint32_t used;  // per stage: filled at least once (thread 0)
};

// One sweep of this block over its bricks (brick b = blockIdx.x + m gridDim.x).
//   sweep A (kB false): stage = s_{n-1} box (buffer cur), res box, flags;
//   sweep B (kB true):  stage = s_n box (buffer cur ^ 1), the brick's res
//     and p, flags.
// Thread 0 keeps ns - 1 bricks in flight ahead of the one computed, reusing a
// stage once all eight warps have arrived on its empty barrier; warps run
// through the bricks without block-wide barriers.  Each warp marches up its
// column with the direction below, at and above its cell in registers
// (sweep A forms s_n = res + bq s_{n-1} where it reads it) and calls
// cell(i, j, k, f, q, A s, s, res, p) for each interior cell (sweep A: A s
// only for cells with maskT, else 0; q = padded index; res and p only in
// sweep B).  Returns false, the same in every thread, after a time-out
// (error recorded).
template <bool kB, class Cell>
__device__ __forceinline__ bool nh_sweep(const NHParams& P, int cur, double bq, unsigned char* smem, NHPipe& pp,
                                         const Cell& cell) {
  const int TY = P.ty, KW = P.kw, KC = P.kc, NS = P.ns, BY = TY + 2, BXY = kNHBoxX * BY;
  const size_t rs = nh_al(nh_rs_bytes(TY, KC)), pb = nh_al(nh_p_bytes(TY, KC)), stage = nh_stage_bytes(TY, KC);
  const size_t fo = nh_flags_off(TY, KC);
  const uint32_t tx_bytes = (uint32_t)(kB ? nh_rs_bytes(TY, KC) + 2 * nh_p_bytes(TY, KC) + nh_f_bytes(TY, KC)
                                          : 2 * nh_rs_bytes(TY, KC) + nh_f_bytes(TY, KC));
  const int nbr = P.nbx * P.nby * P.nbz;
  const int nx = P.G.g.nx, ny = P.G.g.ny, nz = P.G.nz;
  const size_t plane = P.G.plane;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int jj = warp % TY, kk0 = (warp / TY) * KW;
  const int nmine = (int)blockIdx.x < nbr ? (nbr - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  // thread 0: put brick number m of this block into stage st once the stage is free
  auto produce = [&](int m, int st) -> bool {
    if (pp.used & (1u << st)) {
      if (!mbar_wait_bounded(&pp.empty[st], (pp.eph >> st) & 1u, P.timeout_ns)) return false;
      pp.eph ^= 1u << st;
    }
    pp.used |= 1u << st;
    const int b = (int)blockIdx.x + m * (int)gridDim.x;
    const int bx = b % P.nbx, t = b / P.nbx, by = t % P.nby, bz = t / P.nby;
    unsigned char* B = smem + (size_t)st * stage;
    fence_proxy_async_smem();
    fence_proxy_async_global();
    mbar_arrive_expect_tx(&pp.full[st], tx_bytes);
    // boxes: padded column of Fortran i0-2 (even, 16-byte aligned), row of j0-1, level index of k0-1;
    // brick arrays: padded column of i0 (even), row of j0, level index of k0
    const int x = 32 * bx + 2, y = TY * by + 1, z = KC * bz - 1;
    const int xb = 32 * bx + 4, yb = TY * by + 2, zb = KC * bz;
    if (!kB) {  // box 0 = s_{n-1}, box 1 = res
      tma_load_3d(B, &P.map_s[cur], x, y, z, &pp.full[st]);
      tma_load_3d(B + rs, &P.map_res, x, y, z, &pp.full[st]);
    } else {  // box 0 = s_n, then the brick's res and p
      tma_load_3d(B, &P.map_s[cur ^ 1], x, y, z, &pp.full[st]);
      tma_load_3d(B + rs, &P.map_res_brick, xb, yb, zb, &pp.full[st]);
      tma_load_3d(B + rs + pb, &P.map_p, xb, yb, zb, &pp.full[st]);
    }
    // flags: column i0-1 (a multiple of 32 bytes), row j0-1, level k0-1
    tma_load_3d(B + fo, &P.map_f, 32 * bx, TY * by, KC * bz, &pp.full[st]);
    return true;
  };
  // a producer time-out stops the copies; the consumers then time out on the stage that never fills
  bool ok = true, prod_ok = true;
  if (threadIdx.x == 0)
    for (int m = 0; m < NS - 1 && m < nmine && prod_ok; m++) prod_ok = produce(m, m);
  for (int m = 0; m < nmine; m++) {
    const int st = m % NS;
    if (threadIdx.x == 0 && prod_ok && m + NS - 1 < nmine) prod_ok = produce(m + NS - 1, (m + NS - 1) % NS);
    const int b = (int)blockIdx.x + m * (int)gridDim.x;
    const int bx = b % P.nbx, t = b / P.nbx, by = t % P.nby, bz = t / P.nby;
    const int i = 1 + 32 * bx + lane, j = 1 + TY * by + jj;
    const bool col = i <= nx && j <= ny;
    // the column's metric factors load while the brick's copy is in flight
    const size_t q2 = col ? P.G.g.at(i, j) : 0;
    const double tE = col ? __ldg(P.op.tE + q2) : 0.0, tW = col ? __ldg(P.op.tW + q2) : 0.0;
    const double tN = col ? __ldg(P.op.tN + j + 1) : 0.0, tS = col ? __ldg(P.op.tS + j + 1) : 0.0;
    // every lane waits, then the warp agrees, so all its lanes leave the loop together
    ok = __all_sync(0xffffffffu, mbar_wait_bounded(&pp.full[st], (pp.fph >> st) & 1u, P.timeout_ns));
    pp.fph ^= 1u << st;
    if (!ok) break;
    unsigned char* B = smem + (size_t)st * stage;
    const double* S = reinterpret_cast<const double*>(B);
    const double* R1 = reinterpret_cast<const double*>(B + rs);       // sweep A: res box; B: the brick's res
    const double* Pb = reinterpret_cast<const double*>(B + rs + pb);  // sweep B: the brick's p
    const uint8_t* F = B + fo;
    // the direction at box index x: sweep A forms s_n = res + rsnew/rsold * p (:189), separately
    // rounded; sweep B reads the stored s_n
    auto sv = [&](int x) { return kB ? S[x] : __dadd_rn(R1[x], __dmul_rn(bq, S[x])); };
    int k = 1 + KC * bz + kk0;
    const int mend = col ? min(KW, nz - k + 1) : 0;
    if (mend > 0) {
      size_t q = (size_t)(k - 1) * plane + q2;
      int cc = ((kk0 + 1) * BY + jj + 1) * kNHBoxX + lane + 2;
      int fl = (kk0 * TY + jj) * 32 + lane;
      double sdn = sv(cc - BXY), sc = sv(cc);
      double tT = __ldg(P.op.tT + k - 1), tB = __ldg(P.op.tB + k - 1);  // vertical factors, one level ahead
#pragma unroll 2
      for (int mm = 0; mm < mend; mm++) {
        const double sup = sv(cc + BXY);
        const uint32_t f = F[fl];
        const double tTn = k < nz ? __ldg(P.op.tT + k) : 0.0, tBn = k < nz ? __ldg(P.op.tB + k) : 0.0;
        if (kB || (f & kNHMaskT)) {
          const double a = nh_row(f, tE, tW, tN, tS, tT, tB, sdn, sv(cc - kNHBoxX), sv(cc - 1), sc, sv(cc + 1),
                                  sv(cc + kNHBoxX), sup);
          cell(i, j, k, f, q, a, sc, kB ? R1[fl] : 0.0, kB ? Pb[fl] : 0.0);
        } else {
          cell(i, j, k, f, q, 0.0, sc, 0.0, 0.0);  // sweep A stores s_n everywhere
        }
        sdn = sc;
        sc = sup;
        tT = tTn;
        tB = tBn;
        k++;
        q += plane;
        cc += BXY;
        fl += 32 * TY;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&pp.empty[st]);
  }
  if (!ok || !prod_ok) atomicExch(&P.ctl->error, PYOMGPU_TIMEOUT);
  return __syncthreads_and(ok && prod_ok) != 0;  // also: every stage is read to the end before the next sweep
}

// Scalar state of congrad_non_hydro's loop (non_hydrostatic.f90:177-242),
// the same in every thread of every block.  The convergence test of
// iteration n needs max|p| of the direction formed after it, so it runs after
// the next iteration's first sweep (after_a).
struct NHCtl {
  enum { kGo = 0, kOk = 1, kErr = 2 };
  double beta = 0, bb = 0, rtol2bb = 0, eps = 0, rtol = 0;
  double betamin = 0, step1 = 0, est = 0, bq = 0, alpha_prev = 0, rr_prev = 0;
  int max_it = 0, n = 0, status = PYOMGPU_OK;

  __device__ int start(double rsold, double bb_, const NHParams& P) {
    beta = rsold;
    bb = bb_;
    rtol = P.rtol;
    rtol2bb = P.rtol * P.rtol * bb;
    eps = P.eps;
    max_it = P.max_it;
    rr_prev = beta;
    if (beta == 0.0) {  // :177
      n = 0;
      return kOk;
    }
    if (max_it < 1) {
      n = 1;
      status = PYOMGPU_MAXITER;
      return kErr;
    }
    n = 1;
    return kGo;
  }
  // after sweep A of iteration n: (s_n, A s_n) and max|s_n| over maskT
  __device__ int after_a(double sAs, double smax, double& alpha) {
    if (n > 1) {  // convergence test of iteration n-1 (:215-226)
      const int m = n - 1;
      const double step = fabs(alpha_prev) * smax;
      if (m == 1) {
        step1 = step;
        est = step;
        if (step < eps) {
          n = m;
          return kOk;
        }
      } else if (step < eps) {
        const double rate = exp(log(step / step1) / (double)(m - 1));
        est = step * rate / (1.0 - rate);
        if (est < eps) {
          n = m;
          return kOk;
        }
      }
      if (est != est) {
        n = m;
        status = PYOMGPU_NAN;
        return kErr;
      }
      if (rtol > 0.0 && (bb > 0.0 ? rr_prev <= rtol2bb : rr_prev == 0.0)) {
        est = sqrt(rr_prev);
        n = m;
        return kOk;
      }
      if (m >= max_it) {  // :228
        n = max_it + 1;
        status = PYOMGPU_MAXITER;
        return kErr;
      }
    }
    if (sAs == 0.0) return kOk;  // :185
    alpha = beta / sAs;
    return kGo;
  }
  // after sweep B of iteration n: rsnew = (res, res) over maskT
  __device__ int after_b(double rsnew, double alpha) {
    bq = rsnew / beta;  // p = res + rsnew/rsold*p (:189)
    beta = rsnew;
    if (n == 1) {  // divergence test (:197-205)
      betamin = fabs(rsnew);
    } else if (n > 2) {
      betamin = fmin(betamin, fabs(rsnew));
      if (fabs(rsnew) > 100.0 * betamin) {
        status = PYOMGPU_DIVERGED;
        return kErr;
      }
    }
    alpha_prev = alpha;
    rr_prev = rsnew;
    ++n;
    return kGo;
  }
  __device__ void finish(int how, CGResult* out) {
    int converged = 0;
    if (how == kOk) {
      converged = 1;
      status = PYOMGPU_OK;
    } else if (est != est) {
      status = PYOMGPU_NAN;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      out->iterations = n;
      out->converged = converged;
      out->status = status;
      out->est = est;
    }
  }
};

template <bool CX, bool CY>
__global__ void __launch_bounds__(kNHThreads, 2) nh_cg_kernel(const __grid_constant__ NHParams P) {
  extern __shared__ __align__(128) unsigned char smem[];
  const NHGeo G = P.G;
  const NHOp op = P.op;
  const int nx = G.g.nx;
  const uint32_t ny = (uint32_t)G.g.ny;
  const uint32_t nch = (uint32_t)(nx + 31) >> 5;
  const uint32_t nunits = nch * ny * (uint32_t)G.nz;
  constexpr int kWarps = kNHThreads / 32;
  const int lane = threadIdx.x & 31;
  const uint32_t gw = blockIdx.x * kWarps + (threadIdx.x >> 5);
  const uint32_t tw = gridDim.x * kWarps;
  const unsigned nb = gridDim.x;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)P.ns * nh_stage_bytes(P.ty, P.kc));
  NHPipe pp{bars, bars + kNHMaxStages, 0u, 0u, 0u};
  unsigned long long epoch = 0;
  double* __restrict__ pnh = P.p;
  double* __restrict__ res = P.res;

  if (threadIdx.x == 0) {
    for (int st = 0; st < P.ns; st++) {
      mbar_init(&pp.full[st], 1);
      mbar_init(&pp.empty[st], kNHThreads / 32);
    }
    fence_mbar_init();
  }
  __syncthreads();

  // ------------------------------------------------------------------ init
  // res = forc - A p (interior), rsold = dot_3D(res, res)  (:163-176)
  {
    double v[2] = {0.0, 0.0};
    for (uint32_t u = gw; u < nunits; u += tw) {
      int i, j, k;
      nh_unit(u, nch, ny, lane, i, j, k);
      if (i > nx) continue;
      const size_t q = G.at(i, j, k);
      const uint32_t f = __ldg(op.flags + op.fidx((int)ny, i, j, k));
      const double a = nh_apply(op, G, i, j, k, f,
                                [&](int di, int dj, int dk) { return __ldcg(pnh + q + nh_off(G, di, dj, dk)); });
      const double fo = P.forc[fidx3(nx, (int)ny, i, j, k)];
      const double r = __dsub_rn(fo, a);
      ptrdiff_t ox, oy;
      nh_copy_offsets<CX, CY>(G.g, i, j, ox, oy);
      nh_put<CX, CY>(res, q, ox, oy, r);
      if (f & kNHMaskT) {
        v[0] += r * r;
        v[1] += fo * fo;
      }
    }
    double out[2];
    block_reduce<2, -1, kNHThreads>(v, out);
    if (threadIdx.x == 0) {
      double* slot = P.slots + (size_t)blockIdx.x * 4;
      slot[0] = out[0];
      slot[1] = out[1];
    }
  }
  if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns, P.stall_extra)) return;
  double red0[2];
  grid_collect<2, -1, kNHThreads>(P.slots, 4, nb, red0);
  NHCtl ctl;
  int how = ctl.start(red0[0], red0[1], P);

  while (how == NHCtl::kGo) {
    const int cur = ctl.n & 1;
    // -------------------------------------------------------------- sweep A
    {
      double* __restrict__ Sn = P.s[cur ^ 1];
      double acc_dot = 0.0, acc_max = 0.0;
      const bool ok = nh_sweep<false>(
          P, cur, ctl.bq, smem, pp,
          [&](int i, int j, int, uint32_t f, size_t q, double a, double sc, double, double) {
            ptrdiff_t ox, oy;
            nh_copy_offsets<CX, CY>(G.g, i, j, ox, oy);
            nh_put<CX, CY>(Sn, q, ox, oy, sc);
            if (f & kNHMaskT) {  // only masked products enter the sums
              acc_dot += sc * a;
              acc_max = fmax(acc_max, fabs(sc));
            }
          });
      if (!ok) return;
      double v[2] = {acc_dot, acc_max}, out[2];
      block_reduce<2, 1, kNHThreads>(v, out);
      if (threadIdx.x == 0) {
        double* slot = P.slots + (size_t)((epoch & 1) * nb + blockIdx.x) * 4;
        slot[0] = out[0];
        slot[1] = out[1];
      }
    }
    const unsigned long long ep_a = epoch;
    if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns)) return;
    double r2[2];
    grid_collect<2, 1, kNHThreads>(P.slots + (size_t)((ep_a & 1) * nb) * 4, 4, nb, r2);
    double alpha = 0.0;
    how = ctl.after_a(r2[0], r2[1], alpha);
    if (how != NHCtl::kGo) break;
    // -------------------------------------------------------------- sweep B
    double acc_r = 0.0;
    const bool ok = nh_sweep<true>(
        P, cur, ctl.bq, smem, pp,
        [&](int i, int j, int, uint32_t f, size_t q, double a, double sc, double rc, double pc) {
          const double r = __dsub_rn(rc, __dmul_rn(alpha, a));  // res = res - alpha*Ap (:188)
          const double d = __dmul_rn(alpha, sc);                // p_non_hydro + alpha*p (:187)
          ptrdiff_t ox, oy;
          nh_copy_offsets<CX, CY>(G.g, i, j, ox, oy);
          pnh[q] = __dadd_rn(pc, d);
          nh_add_halo<CX, CY>(pnh, q, ox, oy, d);
          nh_put<CX, CY>(res, q, ox, oy, r);
          if (f & kNHMaskT) acc_r += r * r;
        });
    if (!ok) return;
    double v[1] = {acc_r}, out[1];
    block_reduce<1, -1, kNHThreads>(v, out);
    if (threadIdx.x == 0) P.slots[(size_t)((epoch & 1) * nb + blockIdx.x) * 4] = out[0];
    const unsigned long long ep_b = epoch;
    if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns)) return;
    double r1[1];
    grid_collect<1, -1, kNHThreads>(P.slots + (size_t)((ep_b & 1) * nb) * 4, 4, nb, r1);
    how = ctl.after_b(r1[0], alpha);
  }
  ctl.finish(how, P.out);
}

// Block-wide reduction whose result every thread receives.
template <int NV, int kMaxSlot, int kThreads>
__device__ __forceinline__ void block_allreduce(const double (&v)[NV], double (&out)[NV]) {
  __shared__ double sh[NV];
  double r[NV];
  block_reduce<NV, kMaxSlot, kThreads>(v, r);
  if (threadIdx.x == 0)
    for (int k = 0; k < NV; k++) sh[k] = r[k];
  __syncthreads();
  for (int k = 0; k < NV; k++) out[k] = sh[k];
  __syncthreads();
}

// Block reduction for kThreads <= 1024: warp shuffles, then warp 0 over the
// warp results; thread 0 gets the result.  Fixed order.
template <int NV, int kMaxSlot, int kThreads>
__device__ __forceinline__ void block_reduce_fast(const double (&v)[NV], double (&out)[NV]) {
  __shared__ double sh[kThreads / 32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    const double r = (k == kMaxSlot) ? warp_max(v[k]) : warp_sum(v[k]);
    if (lane == 0) sh[w][k] = r;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double r = lane < kThreads / 32 ? sh[lane][k] : 0.0;
      r = (k == kMaxSlot) ? warp_max(r) : warp_sum(r);
      out[k] = r;
    }
  }
  __syncthreads();
}

// Small grids: the whole solve in one thread-block cluster of C <= 16 blocks
// (one per SM).  The interior cells, in compact (i, j, k) order, are split
// into C contiguous chunks; each block keeps res, the direction (two buffers:
// the previous and the one being formed), p_non_hydro and the flags of its
// chunk in shared memory (33 bytes per cell; p is written back at the end,
// the cyclic halo copies of p are summed in global memory as the reference
// sums them) and reads a neighbour in another chunk from the
// owner's shared memory (distributed shared memory).  Sweep A forms the new
// direction res + bq s_old itself wherever it reads it, local or remote, so
// no barrier is needed before its stencil.  A neighbour across a cyclic
// boundary wraps; one across a closed boundary reads 0, as the reference's
// zero halo of p does.  Two cluster
// barriers per iteration carry the reductions; each block's warp 0 combines
// the C block partials in the same order.  Same control flow and per-cell
// arithmetic as nh_cg_kernel.
template <bool CX, bool CY>
__global__ void __launch_bounds__(kNHSmallThreads, 1) nh_cg_small_kernel(const __grid_constant__ NHParams P) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double part[4], total[4];
  __shared__ const double* rankR[kNHMaxCluster];
  __shared__ double* rankS[2][kNHMaxCluster];
  cg::cluster_group cluster = cg::this_cluster();
  const NHGeo G = P.G;
  const NHOp op = P.op;
  const int nx = G.g.nx, ny = G.g.ny, nz = G.nz;
  const int nxy = nx * ny, N = nxy * nz;
  const int C = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
  const int chunk = P.small_chunk;
  const int c0 = rank * chunk, c1 = min(N, c0 + chunk);
  double* R = reinterpret_cast<double*>(smem);
  double* S0 = R + chunk;
  double* S1 = S0 + chunk;
  double* Pl = S1 + chunk;  // p_non_hydro of the chunk
  uint8_t* F = reinterpret_cast<uint8_t*>(Pl + chunk);
  double* __restrict__ pnh = P.p;
  if (threadIdx.x < C) {
    rankR[threadIdx.x] = cluster.map_shared_rank(R, (int)threadIdx.x);
    rankS[0][threadIdx.x] = cluster.map_shared_rank(S0, (int)threadIdx.x);
    rankS[1][threadIdx.x] = cluster.map_shared_rank(S1, (int)threadIdx.x);
  }
  auto decode = [&](int c, int& i, int& j, int& k) {
    i = c % nx + 1;
    const int r = c / nx;
    j = r % ny + 1;
    k = r / ny + 1;
  };
  // compact neighbour of cell c (i, j) in direction (di, dj, dk); -1 across a closed boundary
  auto nbi = [&](int c, int i, int j, int di, int dj, int dk) -> int {
    if (di == 1) return i < nx ? c + 1 : (CX ? c - (nx - 1) : -1);
    if (di == -1) return i > 1 ? c - 1 : (CX ? c + (nx - 1) : -1);
    if (dj == 1) return j < ny ? c + nx : (CY ? c - nx * (ny - 1) : -1);
    if (dj == -1) return j > 1 ? c - nx : (CY ? c + nx * (ny - 1) : -1);
    return c + dk * nxy;  // only read where the vertical face is open, so inside
  };
  // Block partials (thread 0 wrote part[0..nv)) summed over the cluster, max
  // for slot max_slot; warp 0 of every block combines them in rank order.
  auto cluster_total = [&](int nv, int max_slot, double* out) {
    cluster.sync();
    if (threadIdx.x < 32) {
      for (int q = 0; q < nv; q++) {
        double v = 0.0;
        if ((int)threadIdx.x < C) v = cluster.map_shared_rank(part, (int)threadIdx.x)[q];
        v = (q == max_slot) ? warp_max(v) : warp_sum(v);
        if (threadIdx.x == 0) total[q] = v;
      }
    }
    __syncthreads();
    for (int q = 0; q < nv; q++) out[q] = total[q];
  };
  // ------------------------------------------------------------------ init
  double red[2];
  {
    double v[2] = {0.0, 0.0};
    for (int c = c0 + (int)threadIdx.x; c < c1; c += kNHSmallThreads) {
      int i, j, k;
      decode(c, i, j, k);
      const size_t q = G.at(i, j, k);
      const uint32_t f = __ldg(op.flags + op.fidx(ny, i, j, k));
      const double a = nh_apply(op, G, i, j, k, f,
                                [&](int di, int dj, int dk) { return pnh[q + nh_off(G, di, dj, dk)]; });
      const double fo = P.forc[fidx3(nx, ny, i, j, k)];
      const double r = __dsub_rn(fo, a);
      R[c - c0] = r;
      S0[c - c0] = 0.0;
      S1[c - c0] = 0.0;
      Pl[c - c0] = pnh[q];
      F[c - c0] = (uint8_t)f;
      if (f & kNHMaskT) {
        v[0] += r * r;
        v[1] += fo * fo;
      }
    }
    double out[2];
    block_reduce_fast<2, -1, kNHSmallThreads>(v, out);
    if (threadIdx.x == 0) {
      part[0] = out[0];
      part[1] = out[1];
    }
    cluster_total(2, -1, red);
  }
  NHCtl ctl;
  int how = ctl.start(red[0], red[1], P);
  while (how == NHCtl::kGo) {
    const int nw = ctl.n & 1;  // buffer the new direction goes to
    double* const* Sold = rankS[nw ^ 1];
    double* Snew = nw ? S1 : S0;
    const double bq = ctl.bq;
    const double* Sold_local = nw ? S0 : S1;
    // s_n at compact cell n: res + rsnew/rsold * p (:189), separately rounded, from its owner's res and
    // s_old (plain shared-memory loads inside the chunk)
    auto sform = [&](int n) -> double {
      if (n >= c0 && n < c1) return __dadd_rn(R[n - c0], __dmul_rn(bq, Sold_local[n - c0]));
      const int o = n / chunk, l = n - o * chunk;
      return __dadd_rn(rankR[o][l], __dmul_rn(bq, Sold[o][l]));
    };
    // ------------------------------------------------------------ sweep A
    double acc[2] = {0.0, 0.0};
    for (int c = c0 + (int)threadIdx.x; c < c1; c += kNHSmallThreads) {
      const uint32_t f = F[c - c0];
      const double sc = __dadd_rn(R[c - c0], __dmul_rn(bq, (nw ? S0 : S1)[c - c0]));
      Snew[c - c0] = sc;
      if (!(f & kNHMaskT)) continue;
      int i, j, k;
      decode(c, i, j, k);
      const double a = nh_apply(op, G, i, j, k, f, [&](int di, int dj, int dk) {
        if (di == 0 && dj == 0 && dk == 0) return sc;
        const int n = nbi(c, i, j, di, dj, dk);
        return n < 0 ? 0.0 : sform(n);
      });
      acc[0] += sc * a;
      acc[1] = fmax(acc[1], fabs(sc));
    }
    double out2[2], rA[2];
    block_reduce_fast<2, 1, kNHSmallThreads>(acc, out2);
    if (threadIdx.x == 0) {
      part[0] = out2[0];
      part[1] = out2[1];
    }
    cluster_total(2, 1, rA);  // also: every block's new direction is complete
    double alpha = 0.0;
    how = ctl.after_a(rA[0], rA[1], alpha);
    if (how != NHCtl::kGo) break;
    // ------------------------------------------------------------ sweep B
    double* const* Sn = rankS[nw];
    double accr[1] = {0.0};
    for (int c = c0 + (int)threadIdx.x; c < c1; c += kNHSmallThreads) {
      const uint32_t f = F[c - c0];
      int i, j, k;
      decode(c, i, j, k);
      const double a = nh_apply(op, G, i, j, k, f, [&](int di, int dj, int dk) {
        const int n = (di == 0 && dj == 0 && dk == 0) ? c : nbi(c, i, j, di, dj, dk);
        if (n < 0) return 0.0;
        if (n >= c0 && n < c1) return (double)Snew[n - c0];
        const int o = n / chunk;
        return Sn[o][n - o * chunk];
      });
      const double sc = Snew[c - c0];
      const double r = __dsub_rn(R[c - c0], __dmul_rn(alpha, a));  // res = res - alpha*Ap (:188)
      const double d = __dmul_rn(alpha, sc);                        // p_non_hydro + alpha*p (:187)
      Pl[c - c0] = __dadd_rn(Pl[c - c0], d);
      if (CX || CY) {  // the halo copies keep their own sums in global memory (few cells)
        ptrdiff_t ox, oy;
        nh_copy_offsets<CX, CY>(G.g, i, j, ox, oy);
        if (ox || oy) nh_add_halo<CX, CY>(pnh, G.at(i, j, k), ox, oy, d);
      }
      R[c - c0] = r;
      if (f & kNHMaskT) accr[0] += r * r;
    }
    double out1[1], rB[1];
    block_reduce_fast<1, -1, kNHSmallThreads>(accr, out1);
    if (threadIdx.x == 0) part[0] = out1[0];
    cluster_total(1, -1, rB);  // also: no block changes res while a neighbour still forms directions from it
    how = ctl.after_b(rB[0], alpha);
  }
  ctl.finish(how, P.out);
  for (int c = c0 + (int)threadIdx.x; c < c1; c += kNHSmallThreads) {
    int i, j, k;
    decode(c, i, j, k);
    pnh[G.at(i, j, k)] = Pl[c - c0];
  }
  cluster.sync();  // no block leaves while another may still read its shared memory
}

const void* nh_cg_small_kernel_ptr(bool cx, bool cy) {
  if (cx) return cy ? (const void*)nh_cg_small_kernel<true, true> : (const void*)nh_cg_small_kernel<true, false>;
  return cy ? (const void*)nh_cg_small_kernel<false, true> : (const void*)nh_cg_small_kernel<false, false>;
}

const void* nh_cg_kernel_ptr(bool cx, bool cy) {
  if (cx) return cy ? (const void*)nh_cg_kernel<true, true> : (const void*)nh_cg_kernel<true, false>;
  return cy ? (const void*)nh_cg_kernel<false, true> : (const void*)nh_cg_kernel<false, false>;
}

namespace {

__global__ void nh_apply_kernel(const NHGeo G, const NHOp op, const double* __restrict__ p, double* __restrict__ res) {
  const int nx = G.g.nx, ny = G.g.ny;
  const size_t ncell = (size_t)nx * ny * G.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ncell; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nx) + 1;
    const size_t r = e / nx;
    const int j = (int)(r % ny) + 1;
    const int k = (int)(r / ny) + 1;
    const size_t q = G.at(i, j, k);
    res[q] = nh_apply(op, G, i, j, k, op.flags[op.fidx(ny, i, j, k)],
                      [&](int di, int dj, int dk) { return p[q + nh_off(G, di, dj, dk)]; });
  }
}

// Fortran (nx+4, ny+4, nz) <-> padded 3-D, whole arrays (halos included).
__global__ void nh_pack_kernel(const NHGeo G, const double* __restrict__ user, double* __restrict__ pad, int dir) {
  const int X = G.g.nx + 2 * kOnx, Y = G.g.ny + 2 * kOnx;
  const size_t n = (size_t)X * Y * G.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int fi = (int)(e % X);
    const size_t r = e / X;
    const int fj = (int)(r % Y);
    const int k = (int)(r / Y);
    const size_t q = (size_t)k * G.plane + (size_t)fj * G.g.pitch + (size_t)(fi + kXOff);
    if (dir == 0)
      pad[q] = user[e];
    else
      const_cast<double*>(user)[e] = pad[q];
  }
}

int grid_for(size_t n) { return (int)std::min<size_t>(4096, std::max<size_t>(1, (n + 255) / 256)); }

// ---- solve_non_hydrostatic step (non_hydrostatic.f90:5-63), Fortran layout -----------------
__device__ __forceinline__ size_t nh_f(const NHGeo& G, int fi, int fj, int k0) {  // 0-based indices
  return (size_t)fi + (size_t)(G.g.nx + 2 * kOnx) * ((size_t)fj + (size_t)(G.g.ny + 2 * kOnx) * (size_t)k0);
}

// w(:,:,k,taup1) = w(tau) + dt_mom*(dw_mix + (1.5+AB_eps) dw(tau) - (0.5+AB_eps) dw(taum1)) * maskW, k < nz (:13-15)
__global__ void nh_w_kernel(const NHStep S) {
  const size_t n = (size_t)(S.G.g.nx + 4) * (S.G.g.ny + 4) * (S.G.nz - 1);
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    S.w[q] = __dadd_rn(S.w_tau[q],
                       __dmul_rn(__dmul_rn(S.dt_mom, __dsub_rn(__dadd_rn(S.dw_mix[q], __dmul_rn(1.5 + S.AB_eps,
                                                                                               S.dw_tau[q])),
                                                               __dmul_rn(0.5 + S.AB_eps, S.dw_taum1[q]))),
                                 (double)S.maskW[q]));
}

// setcyclic_xyz (parallel_none.f90:188-211) of up to three arrays: every halo position the reference
// fills takes the interior value it ends up with (x copies, then y copies over the x-filled rows).
__global__ void nh_setcyclic_kernel(const NHGeo G, double* a, double* b, double* c) {
  const int X = G.g.nx + 4, Y = G.g.ny + 4;
  const size_t n = (size_t)X * Y * G.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int fi = (int)(e % X);
    const size_t r = e / X;
    const int fj = (int)(r % Y);
    const int k0 = (int)(r / Y);
    int si = fi, sj = fj;  // Fortran index = 0-based index - 1
    if (G.g.cyclic_x) {
      if (fi - 1 > G.g.nx) si = fi - G.g.nx;
      else if (fi - 1 < 1) si = fi + G.g.nx;
    }
    if (G.g.cyclic_y) {
      if (fj - 1 > G.g.ny) sj = fj - G.g.ny;
      else if (fj - 1 < 1) sj = fj + G.g.ny;
    }
    if (si == fi && sj == fj) continue;
    const size_t src = nh_f(G, si, sj, k0);
    for (double* x : {a, b, c})
      if (x) x[e] = x[src];
  }
}

// forc = (div_h(u, v) + dw/dz) / dt_mom on the interior (:25-36); p(taup1) = 2 p(tau) - p(taum1) (:40)
__global__ void nh_forc_kernel(const NHStep S) {
  const int nx = S.G.g.nx, ny = S.G.g.ny, X = nx + 4;
  const size_t n = (size_t)X * (ny + 4) * S.G.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    S.p1[e] = __dsub_rn(2.0 * S.p0[e], S.pm[e]);
    const int fi = (int)(e % X);
    const size_t r = e / X;
    const int fj = (int)(r % (ny + 4));
    const int k0 = (int)(r / (ny + 4));
    const int i = fi - 1, j = fj - 1;  // Fortran indices
    if (i < 1 || i > nx || j < 1 || j > ny) {
      S.forc[e] = 0.0;
      continue;
    }
    const double cj = S.cost[fj];
    double f = __dadd_rn(__ddiv_rn(__dsub_rn(S.u[e], S.u[e - 1]), __dmul_rn(cj, S.dxt[fi])),
                         __ddiv_rn(__dsub_rn(__dmul_rn(S.cosu[fj], S.v[e]), __dmul_rn(S.cosu[fj - 1], S.v[e - X])),
                                   __dmul_rn(cj, S.dyt[fj])));
    const size_t pl = (size_t)X * (ny + 4);
    const double wt = k0 == 0 ? S.w[e] : __dsub_rn(S.w[e], S.w[e - pl]);
    f = __dadd_rn(f, __ddiv_rn(wt, S.dzt[k0]));
    S.forc[e] = __ddiv_rn(f, S.dt_mom);
  }
}

// u, v -= dt_mom * grad p (interior), w -= dt_mom * dp/dz * maskW (whole levels k < nz)  (:52-61)
__global__ void nh_correct_kernel(const NHStep S) {
  const int nx = S.G.g.nx, ny = S.G.g.ny, X = nx + 4;
  const size_t pl = (size_t)X * (ny + 4);
  const size_t n = pl * S.G.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int fi = (int)(e % X);
    const size_t r = e / X;
    const int fj = (int)(r % (ny + 4));
    const int k0 = (int)(r / (ny + 4));
    const int i = fi - 1, j = fj - 1;
    if (i >= 1 && i <= nx && j >= 1 && j <= ny) {
      const double dpx = __dsub_rn(S.p1[e + 1], S.p1[e]);
      S.u[e] = __dsub_rn(S.u[e], __dmul_rn(__ddiv_rn(__dmul_rn(S.dt_mom, dpx), __dmul_rn(S.dxu[fi], S.cost[fj])),
                                           (double)S.maskU[e]));
      const double dpy = __dsub_rn(S.p1[e + X], S.p1[e]);
      S.v[e] = __dsub_rn(S.v[e], __dmul_rn(__ddiv_rn(__dmul_rn(S.dt_mom, dpy), S.dyu[fj]), (double)S.maskV[e]));
    }
    if (k0 < S.G.nz - 1) {
      const double dpz = __dsub_rn(S.p1[e + pl], S.p1[e]);
      S.w[e] = __dsub_rn(S.w[e], __dmul_rn(__ddiv_rn(__dmul_rn(S.dt_mom, dpz), S.dzw[k0]), (double)S.maskW[e]));
    }
  }
}

}  // namespace

void launch_nh_step_pre(const NHStep& S, cudaStream_t st) {
  const size_t n = (size_t)(S.G.g.nx + 4) * (S.G.g.ny + 4) * S.G.nz;
  nh_w_kernel<<<grid_for(n), 256, 0, st>>>(S);
  if (S.G.g.cyclic_x || S.G.g.cyclic_y) nh_setcyclic_kernel<<<grid_for(n), 256, 0, st>>>(S.G, S.u, S.v, S.w);
  nh_forc_kernel<<<grid_for(n), 256, 0, st>>>(S);
}
void launch_nh_step_post(const NHStep& S, cudaStream_t st) {
  const size_t n = (size_t)(S.G.g.nx + 4) * (S.G.g.ny + 4) * S.G.nz;
  if (S.G.g.cyclic_x || S.G.g.cyclic_y) nh_setcyclic_kernel<<<grid_for(n), 256, 0, st>>>(S.G, S.p1, nullptr, nullptr);
  nh_correct_kernel<<<grid_for(n), 256, 0, st>>>(S);
}

void launch_nh_apply(const NHGeo& G, const NHOp& op, const double* p, double* res, cudaStream_t st) {
  nh_apply_kernel<<<grid_for((size_t)G.g.nx * G.g.ny * G.nz), 256, 0, st>>>(G, op, p, res);
}
void launch_nh_pack(const NHGeo& G, const double* user, double* padded, cudaStream_t st) {
  const size_t n = (size_t)(G.g.nx + 4) * (G.g.ny + 4) * G.nz;
  nh_pack_kernel<<<grid_for(n), 256, 0, st>>>(G, user, padded, 0);
}
void launch_nh_unpack(const NHGeo& G, const double* padded, double* user, cudaStream_t st) {
  const size_t n = (size_t)(G.g.nx + 4) * (G.g.ny + 4) * G.nz;
  nh_pack_kernel<<<grid_for(n), 256, 0, st>>>(G, user, const_cast<double*>(padded), 1);
}

}  // namespace pyomgpu

// ===========================================================================
// C ABI
// ===========================================================================
using namespace pyomgpu;

struct pyomgpu_nh {
  int device = 0, nsm = 0;
  NHGeo G{};
  NHOp op{};
  int cyclic_x = 0, cyclic_y = 0;
  size_t nf = 0;  // Fortran-layout elements (nx+4)(ny+4)nz
  uint8_t* flags = nullptr;
  double *tE = nullptr, *tW = nullptr, *tN = nullptr, *tS = nullptr, *tT = nullptr, *tB = nullptr;
  // grid arrays of the full step (solve_non_hydrostatic)
  double *dxt = nullptr, *dxu = nullptr, *dyt = nullptr, *dyu = nullptr, *cost = nullptr, *cosu = nullptr;
  double *dzt = nullptr, *dzw = nullptr;
  uint8_t *mU = nullptr, *mV = nullptr, *mW = nullptr;
  double *p = nullptr, *res = nullptr, *s[2] = {}, *stage_f = nullptr, *stage_p = nullptr;
  SyncCtl* ctl = nullptr;
  double* slots = nullptr;
  CGResult* d_result = nullptr;
  CGResult* h_result = nullptr;
  int* h_err = nullptr;
  int max_blocks = 0;  // slots reserved for this many blocks
  int grid = 0;        // 0: automatic
  int ty = 0, kc = 0;  // brick shape (0: automatic)
  int ns = 0;          // pipeline stages (0: automatic)
  int variant = 0;     // 0 automatic, 1 brick kernel, 2 single-block kernel
  double timeout_s = 2.0;
  unsigned stall_next = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~pyomgpu_nh() {
    void* ptrs[] = {flags, tE, tW, tN, tS, tT, tB, dxt, dxu, dyt, dyu, cost, cosu, dzt, dzw, mU, mV, mW,
                    p, res, s[0], s[1], stage_f, stage_p, ctl, slots,
                    d_result};
    for (void* q : ptrs)
      if (q) cudaFree(q);
    if (h_result) cudaFreeHost(h_result);
    if (h_err) cudaFreeHost(h_err);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

namespace {

int nfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  pyomgpu::set_last_error(buf);
  return code;
}

#define NCK(call)                                                                                       \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      return nfail(PYOMGPU_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
  } while (0)

bool nh_on_device(const void* q) {
  if (!q) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
int nalloc(T** q, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)q, n * sizeof(T));
  if (e != cudaSuccess) return nfail(PYOMGPU_ENOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
  return 0;
}

template <typename T>
int nupload(T** d, const std::vector<T>& h) {
  if (int rc = nalloc(d, h.size())) return rc;
  NCK(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// Fortran-layout input: device pointers pass through, host memory is copied
// into `stage`.
int nh_stage(pyomgpu_nh* h, const double* user, double* stage, const double** out, cudaStream_t st) {
  if (nh_on_device(user)) {
    *out = user;
    return 0;
  }
  NCK(cudaMemcpyAsync(stage, user, h->nf * sizeof(double), cudaMemcpyHostToDevice, st));
  *out = stage;
  return 0;
}

}  // namespace

extern "C" {

int32_t pyomgpu_nh_create(const pyomgpu_grid3d* gr, pyomgpu_nh** out) {
  if (!gr || !out) return nfail(PYOMGPU_EINVAL, "nh_create: null argument");
  *out = nullptr;
  const int nx = gr->nx, ny = gr->ny, nz = gr->nz;
  if (gr->onx != 2) return nfail(PYOMGPU_EINVAL, "nh_create: onx must be 2");
  if (nx < 4 || ny < 1 || nz < 2)
    return nfail(PYOMGPU_EINVAL, "nh_create: need nx >= 4, ny >= 1, nz >= 2 (make_coeff_non_hydro reads maskW(nz-1))");
  if (gr->enable_cyclic_y && ny < 4) return nfail(PYOMGPU_EINVAL, "nh_create: cyclic y needs ny >= 4");
  if (!gr->dxt || !gr->dxu || !gr->dyt || !gr->dyu || !gr->cost || !gr->cosu || !gr->dzt || !gr->dzw ||
      !gr->maskT || !gr->maskU || !gr->maskV || !gr->maskW)
    return nfail(PYOMGPU_EINVAL, "nh_create: every grid array is required");
  const size_t X = nx + 4, Y = ny + 4;
  const size_t ncell = (size_t)nx * ny * nz;
  if ((ncell + 31) / 32 + (size_t)ny * nz > 0xffffffffull / 2)
    return nfail(PYOMGPU_EINVAL, "nh_create: grid too large");
  auto* h = new pyomgpu_nh();
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device);
  h->cyclic_x = gr->enable_cyclic_x != 0;
  h->cyclic_y = gr->enable_cyclic_y != 0;
  Geo g{};
  g.nx = nx;
  g.ny = ny;
  g.pitch = (int)(((X + kXOff) + 31) / 32 * 32);
  g.cyclic_x = h->cyclic_x;
  g.cyclic_y = h->cyclic_y;
  h->G.g = g;
  h->G.nz = nz;
  h->G.plane = g.size();
  h->nf = X * Y * (size_t)nz;
  const size_t np = h->G.size();

  // ---- tables and flags, make_coeff_non_hydro's arithmetic (host IEEE double)
  auto F3 = [&](const double* a, int i, int j, int k) {  // Fortran (i,j,k), 1-based k
    return a[(size_t)(i + 1) + X * ((size_t)(j + 1) + Y * (size_t)(k - 1))];
  };
  auto I1 = [](int i) { return (size_t)(i + 1); };  // Fortran index -> [n+4] array index
  std::vector<double> tE(g.size(), 0.0), tW(g.size(), 0.0), tN(Y, 0.0), tS(Y, 0.0), tT(nz, 0.0), tB(nz, 0.0);
  const int fx = (nx + 31) / 32 * 32;
  std::vector<uint8_t> flags((size_t)fx * ny * nz, 0);
  int bad_mask = 0;
  for (int j = 1; j <= ny; j++) {
    const double c2 = gr->cost[I1(j)] * gr->cost[I1(j)];
    for (int i = 1; i <= nx; i++) {
      tE[g.at(i, j)] = 1.0 / gr->dxu[I1(i)] / gr->dxt[I1(i)] / c2;
      tW[g.at(i, j)] = 1.0 / gr->dxu[I1(i - 1)] / gr->dxt[I1(i)] / c2;
    }
    tN[I1(j)] = 1.0 / gr->dyu[I1(j)] / gr->dyt[I1(j)] * gr->cosu[I1(j)] / gr->cost[I1(j)];
    tS[I1(j)] = 1.0 / gr->dyu[I1(j - 1)] / gr->dyt[I1(j)] * gr->cosu[I1(j - 1)] / gr->cost[I1(j)];
  }
  for (int k = 1; k <= nz; k++) {
    if (k < nz) tT[k - 1] = 1.0 / gr->dzw[k - 1] / gr->dzt[k - 1];
    if (k > 1) tB[k - 1] = 1.0 / gr->dzw[k - 2] / gr->dzt[k - 1];
  }
  auto bit = [&](double m, uint32_t b) -> uint32_t {
    if (m == 1.0) return b;
    if (m != 0.0) bad_mask = 1;
    return 0u;
  };
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        uint32_t f = 0;
        f |= bit(F3(gr->maskU, i, j, k), kNHE);
        f |= bit(F3(gr->maskU, i - 1, j, k), kNHW);
        f |= bit(F3(gr->maskV, i, j, k), kNHN);
        f |= bit(F3(gr->maskV, i, j - 1, k), kNHS);
        if (k < nz) f |= bit(F3(gr->maskW, i, j, k), kNHT);
        if (k > 1) f |= bit(F3(gr->maskW, i, j, k - 1), kNHB);
        f |= bit(F3(gr->maskT, i, j, k), kNHMaskT);
        flags[((size_t)(k - 1) * ny + (j - 1)) * fx + (i - 1)] = (uint8_t)f;
      }
  for (const double* m : {gr->maskT, gr->maskU, gr->maskV, gr->maskW})
    for (size_t q = 0; q < h->nf; q++)
      if (m[q] != 0.0 && m[q] != 1.0) bad_mask = 1;
  if (bad_mask) {
    delete h;
    return nfail(PYOMGPU_EINVAL, "nh_create: masks must hold only 0 and 1");
  }
  int rc = 0;
  if ((rc = nupload(&h->flags, flags)) || (rc = nupload(&h->tE, tE)) || (rc = nupload(&h->tW, tW)) ||
      (rc = nupload(&h->tN, tN)) || (rc = nupload(&h->tS, tS)) || (rc = nupload(&h->tT, tT)) ||
      (rc = nupload(&h->tB, tB)) || (rc = nalloc(&h->p, np)) || (rc = nalloc(&h->res, np)) ||
      (rc = nalloc(&h->s[0], np)) || (rc = nalloc(&h->s[1], np)) ||
      (rc = nalloc(&h->stage_f, h->nf)) || (rc = nalloc(&h->stage_p, h->nf)) || (rc = nalloc(&h->ctl, 1)) ||
      (rc = nalloc(&h->d_result, 1))) {
    delete h;
    return rc;
  }
  {
    auto v1 = [](const double* a, size_t n) { return std::vector<double>(a, a + n); };
    auto m8 = [&](const double* a) {
      std::vector<uint8_t> m(h->nf);
      for (size_t q = 0; q < h->nf; q++) m[q] = a[q] == 1.0 ? 1 : 0;
      return m;
    };
    if ((rc = nupload(&h->dxt, v1(gr->dxt, X))) || (rc = nupload(&h->dxu, v1(gr->dxu, X))) ||
        (rc = nupload(&h->dyt, v1(gr->dyt, Y))) || (rc = nupload(&h->dyu, v1(gr->dyu, Y))) ||
        (rc = nupload(&h->cost, v1(gr->cost, Y))) || (rc = nupload(&h->cosu, v1(gr->cosu, Y))) ||
        (rc = nupload(&h->dzt, v1(gr->dzt, nz))) || (rc = nupload(&h->dzw, v1(gr->dzw, nz))) ||
        (rc = nupload(&h->mU, m8(gr->maskU))) || (rc = nupload(&h->mV, m8(gr->maskV))) ||
        (rc = nupload(&h->mW, m8(gr->maskW)))) {
      delete h;
      return rc;
    }
  }
  h->op = NHOp{h->flags, h->tE, h->tW, h->tN, h->tS, h->tT, h->tB, fx};
  if (cudaMemset(h->p, 0, np * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return nfail(PYOMGPU_ECUDA, "nh_create: cudaMemset");
  }
  bool attr_ok = true;
  for (int v = 0; v < 4; v++)
    attr_ok = attr_ok && cudaFuncSetAttribute(nh_cg_kernel_ptr(v & 1, v >> 1),
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kNHSmemMax) == cudaSuccess;
  for (int v = 0; v < 4; v++)
    attr_ok = attr_ok &&
              cudaFuncSetAttribute(nh_cg_small_kernel_ptr(v & 1, v >> 1), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kNHSmallSmemMax) == cudaSuccess &&
              cudaFuncSetAttribute(nh_cg_small_kernel_ptr(v & 1, v >> 1),
                                   cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
  if (!attr_ok) {
    cudaGetLastError();
    delete h;
    return nfail(PYOMGPU_ECUDA, "nh_create: shared-memory attribute");
  }
  h->max_blocks = 4 * kNHThreads;  // grid_collect reads <= 4 slots per thread
  if ((rc = nalloc(&h->slots, (size_t)2 * h->max_blocks * 4))) {
    delete h;
    return rc;
  }
  if (cudaMallocHost((void**)&h->h_result, sizeof(CGResult)) != cudaSuccess ||
      cudaMallocHost((void**)&h->h_err, sizeof(int)) != cudaSuccess || cudaEventCreate(&h->e0) != cudaSuccess ||
      cudaEventCreate(&h->e1) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return nfail(PYOMGPU_ECUDA, "nh_create: host buffers / events");
  }
  *out = h;
  return PYOMGPU_OK;
}

void pyomgpu_nh_destroy(pyomgpu_nh* h) { delete h; }

int32_t pyomgpu_nh_set_sync_timeout(pyomgpu_nh* h, double seconds) {
  if (!h || !(seconds > 0)) return nfail(PYOMGPU_EINVAL, "nh_set_sync_timeout: bad argument");
  h->timeout_s = seconds;
  return PYOMGPU_OK;
}

int32_t pyomgpu_nh_inject_barrier_stall(pyomgpu_nh* h, int32_t enable) {
  if (!h) return nfail(PYOMGPU_EINVAL, "nh_inject_barrier_stall: null handle");
  h->stall_next = enable ? 1u : 0u;
  return PYOMGPU_OK;
}

int32_t pyomgpu_nh_set_grid(pyomgpu_nh* h, int32_t blocks) {
  if (!h || blocks < 0) return nfail(PYOMGPU_EINVAL, "nh_set_grid: bad argument");
  h->grid = std::min(blocks, h->max_blocks);
  return PYOMGPU_OK;
}

int32_t pyomgpu_nh_set_brick(pyomgpu_nh* h, int32_t ty, int32_t kc) {
  if (!h || ty < 0 || kc < 0 || (ty > 0) != (kc > 0))
    return nfail(PYOMGPU_EINVAL, "nh_set_brick: ty and kc both positive (or both 0 = automatic)");
  if (ty > 0 && ((ty != 1 && ty != 2 && ty != 4 && ty != 8) || kc % (8 / ty) != 0 || kc > 248 ||
                 nh_smem_bytes(ty, kc, 2) > kNHSmemMax))
    return nfail(PYOMGPU_EINVAL,
                 "nh_set_brick: ty in {1,2,4,8}, kc a multiple of 8/ty, and the staged boxes within shared memory");
  h->ty = ty;
  h->kc = kc;
  return PYOMGPU_OK;
}

int32_t pyomgpu_nh_set_stages(pyomgpu_nh* h, int32_t stages) {
  if (!h || stages < 0 || stages == 1 || stages > kNHMaxStages)
    return nfail(PYOMGPU_EINVAL, "nh_set_stages: 2..%d stages (0 = automatic)", kNHMaxStages);
  h->ns = stages;
  return PYOMGPU_OK;
}

int32_t pyomgpu_nh_set_variant(pyomgpu_nh* h, int32_t variant) {
  if (!h || variant < 0 || variant > 2) return nfail(PYOMGPU_EINVAL, "nh_set_variant: 0, 1 or 2");
  if (variant == 2 && (size_t)h->G.g.nx * h->G.g.ny * h->G.nz > (size_t)kNHSmallMaxCells)
    return nfail(PYOMGPU_EINVAL, "nh_set_variant: the cluster kernel holds at most %d cells", kNHSmallMaxCells);
  h->variant = variant;
  return PYOMGPU_OK;
}

int32_t pyomgpu_apply_op_3d(pyomgpu_nh* h, const double* p1, double* res, pyomgpu_stream stream) {
  if (!h || !p1 || !res) return nfail(PYOMGPU_EINVAL, "apply_op_3d: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const double* pin = nullptr;
  if (int rc = nh_stage(h, p1, h->stage_p, &pin, st)) return rc;
  const size_t bytes = h->G.size() * sizeof(double);
  launch_nh_pack(h->G, pin, h->p, st);
  NCK(cudaMemsetAsync(h->res, 0, bytes, st));
  launch_nh_apply(h->G, h->op, h->p, h->res, st);
  const bool dev_out = nh_on_device(res);
  double* dst = dev_out ? res : h->stage_f;
  launch_nh_unpack(h->G, h->res, dst, st);
  NCK(cudaGetLastError());
  if (!dev_out) NCK(cudaMemcpyAsync(res, h->stage_f, h->nf * sizeof(double), cudaMemcpyDeviceToHost, st));
  NCK(cudaStreamSynchronize(st));
  return PYOMGPU_OK;
}

}  // extern "C"

namespace {

int nh_finish_cg(pyomgpu_nh* h, double* pdev, pyomgpu_solve_info* info, cudaStream_t st);

// congrad_non_hydro on device arrays: fdev (forcing) and pdev (p_non_hydro(:,:,:,taup1), in/out), both
// Fortran layout.  pdev may be a staging buffer whose result the caller copies out.
int nh_run_cg(pyomgpu_nh* h, const double* fdev, double* pdev, double eps, int max_it, pyomgpu_solve_info* info,
              cudaStream_t st) {
  const size_t bytes = h->G.size() * sizeof(double);
  launch_nh_pack(h->G, pdev, h->p, st);
  for (double* b : {h->res, h->s[0], h->s[1]}) NCK(cudaMemsetAsync(b, 0, bytes, st));
  NCK(cudaMemsetAsync(h->ctl, 0, sizeof(SyncCtl), st));
  NHParams P{};
  P.G = h->G;
  P.op = h->op;
  P.forc = fdev;
  P.p = h->p;
  P.res = h->res;
  P.s[0] = h->s[0];
  P.s[1] = h->s[1];
  P.eps = eps;
  P.max_it = max_it;
  P.rtol = 0.0;
  P.ctl = h->ctl;
  P.slots = h->slots;
  P.timeout_ns = (unsigned long long)(h->timeout_s * 1e9);
  P.stall_extra = h->stall_next;
  h->stall_next = 0;
  P.out = h->d_result;
  const size_t ncell = (size_t)h->G.g.nx * h->G.g.ny * h->G.nz;
  const bool small = h->variant == 2 || (h->variant == 0 && ncell <= (size_t)kNHClusterAuto);
  if (small) {
    // cluster of C = 1, 2, 4, 8 or 16 blocks with about one cell per thread, each chunk within shared memory
    int C = 1;
    while (C < kNHMaxCluster && ((size_t)C * kNHSmallThreads < ncell || (ncell + C - 1) / C > (size_t)kNHSmallMaxChunk))
      C *= 2;
    const int chunk = (int)((ncell + C - 1) / C);
    P.small_chunk = chunk;
    const void* kfs = nh_cg_small_kernel_ptr(h->cyclic_x != 0, h->cyclic_y != 0);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kNHSmallThreads);
    cfg.dynamicSmemBytes = nh_small_smem_bytes(chunk);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kfs, &cfg) != cudaSuccess) {
      cudaGetLastError();
      nclusters = 0;
    }
    if (nclusters >= 1) {
      void* sargs[] = {&P};
      NCK(cudaEventRecord(h->e0, st));
      NCK(cudaLaunchKernelExC(&cfg, kfs, sargs));
      NCK(cudaEventRecord(h->e1, st));
      return nh_finish_cg(h, pdev, info, st);
    }
    if (h->variant == 2) return nfail(PYOMGPU_ECUDA, "congrad_non_hydro: a cluster of %d blocks cannot be placed", C);
    // automatic choice: the brick kernel below
  }
  // brick shape: 32 x ty x kc, ty the largest power of two <= min(8, ny), kc = (8/ty) kw with kw the
  // largest level count per warp whose pipeline stages leave room for two blocks per SM
  int ty = h->ty, kc = h->kc, ns = h->ns > 0 ? h->ns : 2;
  if (ty == 0) {
    ty = h->G.g.ny >= 8 ? 8 : h->G.g.ny >= 4 ? 4 : h->G.g.ny >= 2 ? 2 : 1;
    const int seg = 8 / ty;
    const int kw_need = (h->G.nz + seg - 1) / seg;
    int kw = 1;
    while (kw < kw_need && nh_smem_bytes(ty, seg * (kw + 1), ns) <= (size_t)113 * 1024) kw++;
    kc = seg * kw;
  }
  while (ns > 2 && nh_smem_bytes(ty, kc, ns) > kNHSmemMax) ns--;
  const size_t smem = nh_smem_bytes(ty, kc, ns);
  if (smem > kNHSmemMax) return nfail(PYOMGPU_EINVAL, "congrad_non_hydro: brick boxes exceed shared memory");
  P.ns = ns;
  P.ty = ty;
  P.kc = kc;
  P.kw = kc / (8 / ty);
  P.nbx = (h->G.g.nx + 31) / 32;
  P.nby = (h->G.g.ny + ty - 1) / ty;
  P.nbz = (h->G.nz + kc - 1) / kc;
  {
    const uint64_t dims[3] = {(uint64_t)h->G.g.pitch, (uint64_t)(h->G.g.ny + 2 * kOnx), (uint64_t)h->G.nz};
    const uint64_t strides[2] = {(uint64_t)h->G.g.pitch * 8, (uint64_t)h->G.plane * 8};
    const uint32_t box[3] = {(uint32_t)kNHBoxX, (uint32_t)(ty + 2), (uint32_t)(kc + 2)};
    const uint32_t pbox[3] = {32u, (uint32_t)ty, (uint32_t)kc};
    const uint64_t fdims[3] = {(uint64_t)h->op.fx, (uint64_t)h->G.g.ny, (uint64_t)h->G.nz};
    const uint64_t fstrides[2] = {(uint64_t)h->op.fx, (uint64_t)h->op.fx * h->G.g.ny};
    int bad = 0;
    bad |= encode_map(&P.map_res, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, h->res, dims, strides, box);
    bad |= encode_map(&P.map_res_brick, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, h->res, dims, strides, pbox);
    for (int b = 0; b < 2; b++)
      bad |= encode_map(&P.map_s[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, h->s[b], dims, strides, box);
    bad |= encode_map(&P.map_p, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, h->p, dims, strides, pbox);
    bad |= encode_map(&P.map_f, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->flags, fdims, fstrides, pbox);
    if (bad) return nfail(PYOMGPU_ECUDA, "congrad_non_hydro: cuTensorMapEncodeTiled failed");
  }
  int per_sm = 0;
  const void* kfn = nh_cg_kernel_ptr(h->cyclic_x != 0, h->cyclic_y != 0);
  NCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kNHThreads, smem));
  if (per_sm < 1) return nfail(PYOMGPU_EINVAL, "congrad_non_hydro: brick does not fit on an SM");
  const int coresident = std::min(per_sm * h->nsm, h->max_blocks);
  const int nbricks = P.nbx * P.nby * P.nbz;
  int grid = h->grid > 0 ? std::min(h->grid, coresident) : std::min(coresident, nbricks);
  grid = std::max(1, grid);
  void* args[] = {&P};
  NCK(cudaEventRecord(h->e0, st));
  NCK(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kNHThreads), args, smem, st));
  NCK(cudaEventRecord(h->e1, st));
  return nh_finish_cg(h, pdev, info, st);
}

// Result of a CG launch: status, iterations, device time; p unpacked to pdev.
int nh_finish_cg(pyomgpu_nh* h, double* pdev, pyomgpu_solve_info* info, cudaStream_t st) {
  NCK(cudaMemcpyAsync(h->h_result, h->d_result, sizeof(CGResult), cudaMemcpyDeviceToHost, st));
  NCK(cudaMemcpyAsync(h->h_err, &h->ctl->error, sizeof(int), cudaMemcpyDeviceToHost, st));
  launch_nh_unpack(h->G, h->p, pdev, st);
  NCK(cudaGetLastError());
  NCK(cudaStreamSynchronize(st));
  const int err = *h->h_err;
  float ms = 0.f;
  NCK(cudaEventElapsedTime(&ms, h->e0, h->e1));
  if (info) {
    info->iterations = h->h_result->iterations;
    info->converged = h->h_result->converged;
    info->status = h->h_result->status;
    info->outer_iterations = 1;
    info->estimated_error = h->h_result->est;
    info->rel_residual = -1.0;
    info->device_ms = ms;
    info->kernel_launches = 1;
    info->fcg_iterations = 0;
    if (err) {
      info->status = PYOMGPU_TIMEOUT;
      info->converged = 0;
    }
  }
  if (err) return nfail(PYOMGPU_TIMEOUT, "grid barrier wait exceeded %.3f s", h->timeout_s);
  return h->h_result->status;
}

}  // namespace

extern "C" {

int32_t pyomgpu_congrad_non_hydro(pyomgpu_nh* h, const double* forc, double* p, double eps, int32_t max_it,
                                  pyomgpu_solve_info* info, pyomgpu_stream stream) {
  if (!h || !forc || !p) return nfail(PYOMGPU_EINVAL, "congrad_non_hydro: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const double* fdev = nullptr;
  if (int rc = nh_stage(h, forc, h->stage_f, &fdev, st)) return rc;
  const bool p_dev = nh_on_device(p);
  if (!p_dev) NCK(cudaMemcpyAsync(h->stage_p, p, h->nf * sizeof(double), cudaMemcpyHostToDevice, st));
  const int rc = nh_run_cg(h, fdev, p_dev ? p : h->stage_p, eps, max_it, info, st);
  if (rc < 0 && rc != PYOMGPU_TIMEOUT) return rc;
  if (!p_dev) {
    NCK(cudaMemcpyAsync(p, h->stage_p, h->nf * sizeof(double), cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
  }
  return rc;
}

int32_t pyomgpu_solve_non_hydrostatic(pyomgpu_nh* h, pyomgpu_state3d* s, pyomgpu_solve_info* info,
                                      pyomgpu_stream stream) {
  if (!h || !s || !s->u || !s->v || !s->w || !s->dw || !s->dw_mix || !s->p_non_hydro)
    return nfail(PYOMGPU_EINVAL, "solve_non_hydrostatic: null argument");
  for (int t : {s->taum1, s->tau, s->taup1})
    if (t < 1 || t > 3) return nfail(PYOMGPU_EINVAL, "solve_non_hydrostatic: time levels are 1..3");
  for (const void* q : {(const void*)s->u, (const void*)s->v, (const void*)s->w, (const void*)s->dw,
                        (const void*)s->dw_mix, (const void*)s->p_non_hydro})
    if (!nh_on_device(q)) return nfail(PYOMGPU_EINVAL, "solve_non_hydrostatic: model arrays must be device memory");
  cudaStream_t st = (cudaStream_t)stream;
  NHStep S{};
  S.G = h->G;
  S.dxt = h->dxt;
  S.dxu = h->dxu;
  S.dyt = h->dyt;
  S.dyu = h->dyu;
  S.cost = h->cost;
  S.cosu = h->cosu;
  S.dzt = h->dzt;
  S.dzw = h->dzw;
  S.maskU = h->mU;
  S.maskV = h->mV;
  S.maskW = h->mW;
  const size_t n3 = h->nf;
  S.u = s->u + (size_t)(s->taup1 - 1) * n3;
  S.v = s->v + (size_t)(s->taup1 - 1) * n3;
  S.w = s->w + (size_t)(s->taup1 - 1) * n3;
  S.w_tau = s->w + (size_t)(s->tau - 1) * n3;
  S.dw_tau = s->dw + (size_t)(s->tau - 1) * n3;
  S.dw_taum1 = s->dw + (size_t)(s->taum1 - 1) * n3;
  S.dw_mix = s->dw_mix;
  S.p1 = s->p_non_hydro + (size_t)(s->taup1 - 1) * n3;
  S.p0 = s->p_non_hydro + (size_t)(s->tau - 1) * n3;
  S.pm = s->p_non_hydro + (size_t)(s->taum1 - 1) * n3;
  S.forc = h->stage_f;
  S.dt_mom = s->dt_mom;
  S.AB_eps = s->AB_eps;
  launch_nh_step_pre(S, st);   // w(taup1), setcyclic u/v/w, forcing, first guess
  NCK(cudaGetLastError());
  const int rc = nh_run_cg(h, h->stage_f, S.p1, s->congr_epsilon_non_hydro, s->congr_max_itts_non_hydro, info, st);
  if (rc < 0) return rc;
  s->congr_itts_non_hydro = info ? info->iterations : h->h_result->iterations;
  launch_nh_step_post(S, st);  // setcyclic p, velocity correction
  if (s->itt == 0) {           // :44-47
    double* p_tau = s->p_non_hydro + (size_t)(s->tau - 1) * n3;
    double* p_taum1 = s->p_non_hydro + (size_t)(s->taum1 - 1) * n3;
    NCK(cudaMemcpyAsync(p_tau, S.p1, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    NCK(cudaMemcpyAsync(p_taum1, S.p1, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  NCK(cudaGetLastError());
  NCK(cudaStreamSynchronize(st));
  return rc;
}

}  // extern "C"
