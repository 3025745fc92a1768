// Persistent work-queue CG: many independent streamfunction solves in one
// launch, each following congrad_streamfunction's control flow
// (solve_streamfct.f90:153-327) with its own scalars.
//
// The tiles of all problems form one task list; every block walks it with a
// static stride.  All problems advance in lockstep through three kinds of
// sweep (init, A: direction + stencil, B: update) separated by grid barriers.
// The last block to reach a barrier sums each problem's per-tile partials in
// a fixed order, runs each problem's stopping logic, and releases the others
// with a generation flag, so every problem ends with exactly the iterations
// and status an individual solve would give.
#include <math.h>

#include "cg_batch.cuh"

namespace pyomgpu {

namespace {

constexpr int kBX = kOnx + 64;  // box columns: Fortran i0-1 .. i0+64
constexpr int kTX = 64, kTY = 16;
constexpr int kBY = kTY + 2;
constexpr int kBoxN = kBX * kBY;

enum : int { kInit = 0, kSweepA = 1, kSweepB = 2 };

__device__ __forceinline__ unsigned long long atom_add_acqrel(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ int task_problem(const BatchParams& P, int task, int p0, int p1) {
  int lo = p0, hi = p1 - 1;  // last problem of the group with tile0 <= task
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P.probs[mid].tile0 <= task)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The state moves through L2 only (ld.cg / st.cg): the reducing block may be
// a different one at every barrier, and a stale L1 line must never be read.
__device__ __forceinline__ BatchState load_state(const BatchState* p) {
  BatchState s;
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(p);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(&s);
#pragma unroll
  for (int k = 0; k < 11; k++) dst[k] = __ldcg(src + k);
  return s;
}
__device__ __forceinline__ void store_state(BatchState* p, const BatchState& s) {
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(p);
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&s);
#pragma unroll
  for (int k = 0; k < 11; k++) __stcg(dst + k, src[k]);
}

// ---------------------------------------------------------------- state logic
__device__ void finish(BatchState& st, bool ok, int status) {
  st.phase = 0;
  st.converged = ok ? 1 : 0;
  st.status = ok ? PYOMGPU_OK : status;
  if (!ok && st.est != st.est) st.status = PYOMGPU_NAN;
}

// top of iteration n (solve_streamfct.f90:223-244)
__device__ void start_iteration(BatchState& st, const BatchProblem& pr, int n) {
  st.n = n;
  if (n > pr.max_it) return finish(st, false, PYOMGPU_MAXITER);  // :303-304
  if (st.beta != st.beta) {  // early NaN stop (the reference runs on and halts at the end)
    st.est = st.beta;
    return finish(st, false, PYOMGPU_NAN);
  }
  if (n == 1) {
    st.betamin = fabs(st.beta);
  } else if (n > 2) {
    st.betamin = fmin(st.betamin, fabs(st.beta));
    if (fabs(st.beta) > 100.0 * st.betamin) return finish(st, false, PYOMGPU_DIVERGED);
  }
  st.bq = st.beta / st.betam1;  // :244
  st.phase = 1;
}

// v = (beta, ||forc||^2, ||res||^2, max|Z res|) of the initial residual
__device__ void after_init(BatchState& st, const BatchProblem& pr, const double* v) {
  st.beta = v[0];
  st.bb = v[1] > 0.0 ? v[1] : v[2];  // the rtol reference: ||forc||, or ||res_0|| for a zero forcing
  st.betam1 = 1.0;
  st.est = 0.0;
  st.stop_after = 0;
  if (100.0 * v[3] < pr.eps) {  // solve_streamfct.f90:210-213
    st.est = 100.0 * v[3];
    st.n = 0;
    return finish(st, true, 0);
  }
  start_iteration(st, pr, 1);
}

// v = ((s, As), max|s|)
__device__ void after_a(BatchState& st, const BatchProblem& pr, const double* v) {
  const double sAs = v[0], smax = v[1];
  if (fabs(sAs) < fabs(st.beta) * (double)1.e-10f) {  // :262-266, a default-real literal
    st.est = 100.0 * smax;
    return finish(st, true, 0);
  }
  st.alpha = st.beta / sAs;
  const double step = fabs(st.alpha) * smax;  // :283-297, applied after the update
  st.stop_after = 0;
  if (st.n == 1) {
    st.step1 = step;
    st.est = step;
    st.stop_after = step < pr.eps;
  } else if (step < pr.eps) {
    const double rate = exp(log(step / st.step1) / (double)(st.n - 1));
    st.est = step * rate / (1.0 - rate);
    st.stop_after = st.est < pr.eps;
  }
  st.phase = 2;
}

// v = ((Z res, res), ||res||^2) of the updated residual
__device__ void after_b(BatchState& st, const BatchProblem& pr, const double* v) {
  if (st.stop_after) return finish(st, true, 0);
  const double bnext = v[0], rr = v[1];
  if (pr.rtol > 0.0 && (st.bb > 0.0 ? rr <= pr.rtol * pr.rtol * st.bb : rr == 0.0)) {
    st.est = sqrt(rr);
    return finish(st, true, 0);
  }
  st.betam1 = st.beta;
  st.beta = bnext;
  start_iteration(st, pr, st.n + 1);
}

// Grid barrier whose last arrival reduces the partials of every problem that
// took part in the sweep just finished and advances its state.  Returns false
// on time-out.
__device__ bool reduce_barrier(const BatchParams& P, unsigned long long& epoch, int kind, int p0, int p1,
                               unsigned extra = 0) {
  __shared__ int s_last, s_ok, s_any;
  __syncthreads();
  epoch += 1;
  if (threadIdx.x == 0) {
    const unsigned long long old = atom_add_acqrel(&P.ctl->arrive, 1ull);
    s_last = (old + 1 == epoch * (unsigned long long)gridDim.x + extra);
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    // every partial of this sweep is visible (acquire side of the arrivals)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int any = 0;
    for (int p = p0 + warp; p < p1; p += kBatchThreads / 32) {
      const BatchProblem& pr = P.probs[p];
      const int phase = __ldcg(&P.state[p].phase);
      if (kind != kInit && phase != kind) {  // finished earlier (init reduces every problem)
        if (lane == 0) any |= phase != 0;
        continue;
      }
      const int nt = pr.ntx * pr.nty;
      const int nv = (kind == kInit) ? 4 : 2;
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      // lane l sums tiles l, l+32, l+64, ... in that order; four tiles' partials are
      // loaded before they are added, so the loads overlap
      for (int t0 = lane; t0 < nt; t0 += 128) {
        double x[4][4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int t = t0 + 32 * u;
          const double* q = P.part + (size_t)(pr.tile0 + (t < nt ? t : 0)) * 4;
#pragma unroll
          for (int k = 0; k < 4; k++) x[u][k] = (t < nt && k < nv) ? __ldcg(q + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (t0 + 32 * u >= nt) break;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            if (k >= nv) break;
            const bool is_max = (kind == kInit && k == 3) || (kind == kSweepA && k == 1);
            v[k] = is_max ? fmax(v[k], x[u][k]) : v[k] + x[u][k];
          }
        }
      }
      for (int k = 0; k < nv; k++) {
        const bool is_max = (kind == kInit && k == 3) || (kind == kSweepA && k == 1);
        v[k] = is_max ? warp_max(v[k]) : warp_sum(v[k]);
      }
      if (lane == 0) {
        BatchState st = load_state(&P.state[p]);
        if (kind == kInit)
          after_init(st, pr, v);
        else if (kind == kSweepA)
          after_a(st, pr, v);
        else
          after_b(st, pr, v);
        store_state(&P.state[p], st);
        any |= st.phase != 0;
      }
    }
    __threadfence();
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    if (lane == 0 && any) atomicOr(&s_any, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      __stcg(P.any_active, s_any);
      __threadfence();
      st_release_u64(P.gen, epoch);
    }
  } else if (threadIdx.x == 0) {
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    while (ld_acquire_u64(P.gen) < epoch) {
      if ((++spins & 63u) == 0u) {
        if (ld_relaxed_i32(&P.ctl->error) != 0 || globaltimer_ns() - t0 > P.timeout_ns) {
          atomicExch(&P.ctl->error, PYOMGPU_TIMEOUT);
          s_ok = 0;
          break;
        }
      }
    }
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace

__global__ void __launch_bounds__(kBatchThreads, 4) cg_batch_kernel(const BatchParams P) {
  __shared__ double b_s[kBoxN], b_FX[kBoxN], b_FY[kBoxN];
  unsigned long long epoch = 0;

  for (int grp = 0; grp < P.ngroup; grp++) {
  const int p0 = P.group[grp], p1 = P.group[grp + 1];
  const int t_lo = P.probs[p0].tile0;
  const int t_hi = P.probs[p1 - 1].tile0 + P.probs[p1 - 1].ntx * P.probs[p1 - 1].nty;
  // ---- init: res = forc - A sol -------------------------------------------------
  for (int task = t_lo + blockIdx.x; task < t_hi; task += gridDim.x) {
    const int p = task_problem(P, task, p0, p1);
    const BatchProblem& pr = P.probs[p];
    const Geo g = pr.g;
    const int lt = task - pr.tile0;
    const int i0 = 1 + kTX * (lt % pr.ntx), j0 = 1 + kTY * (lt / pr.ntx);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int e = threadIdx.x; e < kTX * kTY; e += kBatchThreads) {
      const int i = i0 + e % kTX, j = j0 + e / kTX;
      if (i > g.nx || j > g.ny) continue;
      const size_t q = g.at(i, j);
      const double f = pr.forc[fidx(g.nx, i, j)];
      const double r = f - apply_point(pr.op, g, pr.sol, i, j);
      store_cyclic(pr.res, g, i, j, r);
      const double w = pr.op.W[q];
      const double zr = w * r;
      const double wd = pr.weighted ? 1.0 / (pr.op.ax[i + 1] * pr.op.by[j + 1]) : 1.0;
      v[0] += (wd * zr) * r;
      if (w != 0.0) {
        v[1] += f * f;
        v[2] += r * r;
      }
      v[3] = fmax(v[3], fabs(zr));
    }
    double out[4];
    block_reduce<4, 3, kBatchThreads>(v, out);
    if (threadIdx.x == 0)
      for (int k = 0; k < 4; k++) P.part[(size_t)task * 4 + k] = out[k];
  }
  if (!reduce_barrier(P, epoch, kInit, p0, p1, grp == 0 ? P.stall_extra : 0u)) return;

  for (;;) {
    if (!__ldcg(P.any_active)) break;
    // ---- sweep A: s_new = Z res + bq s_old on tile + halo, As = A s_new ---------------
    for (int task = t_lo + blockIdx.x; task < t_hi; task += gridDim.x) {
      const int p = task_problem(P, task, p0, p1);
      if (__ldcg(&P.state[p].phase) != 1) continue;
      const BatchProblem& pr = P.probs[p];
      const Geo g = pr.g;
      const OpDev<double> op = pr.op;
      const int n = __ldcg(&P.state[p].n);
      const double bq = __ldcg(&P.state[p].bq);
      const double* __restrict__ so = pr.s[(n + 1) & 1];
      double* __restrict__ sn = pr.s[n & 1];
      const int lt = task - pr.tile0;
      const int i0 = 1 + kTX * (lt % pr.ntx), j0 = 1 + kTY * (lt / pr.ntx);
      __syncthreads();  // shared boxes of the previous task are free
      // four box points per thread in flight (the loads do not depend on the shared stores)
#pragma unroll 4
      for (int e = threadIdx.x; e < kBoxN; e += kBatchThreads) {
        const int i = i0 - 1 + e % kBX, j = j0 - 1 + e / kBX;
        double r = 0.0, w = 0.0, s = 0.0, fx = 0.0, fy = 0.0;
        if (i <= g.nx + kOnx && j <= g.ny + kOnx) {
          const size_t q = g.at(i, j);
          r = pr.res[q];
          w = op.W[q];
          s = so[q];
          fx = op.FX[q];
          fy = op.FY[q];
        }
        b_s[e] = w * r + bq * s;
        b_FX[e] = fx;
        b_FY[e] = fy;
      }
      __syncthreads();
      double v[2] = {0.0, 0.0};
      for (int e = threadIdx.x; e < kTX * kTY; e += kBatchThreads) {
        const int c = e % kTX, rr = e / kTX;
        const int i = i0 + c, j = j0 + rr;
        if (i > g.nx || j > g.ny) continue;
        const int k = (rr + 1) * kBX + c + 1;
        const double sc = b_s[k];
        const double a = op.ax[i + 1] * op.bx[j + 1] * (b_FX[k + 1] * (b_s[k + 1] - sc) + b_FX[k] * (b_s[k - 1] - sc)) +
                         op.by[j + 1] * (b_FY[k + kBX] * (b_s[k + kBX] - sc) + b_FY[k] * (b_s[k - kBX] - sc));
        store_cyclic(sn, g, i, j, sc);
        pr.As[g.at(i, j)] = a;
        const double wd = pr.weighted ? 1.0 / (op.ax[i + 1] * op.by[j + 1]) : 1.0;
        v[0] += (wd * sc) * a;
        v[1] = fmax(v[1], fabs(sc));
      }
      double out[2];
      block_reduce<2, 1, kBatchThreads>(v, out);
      if (threadIdx.x == 0) {
        P.part[(size_t)task * 4] = out[0];
        P.part[(size_t)task * 4 + 1] = out[1];
      }
    }
    if (!reduce_barrier(P, epoch, kSweepA, p0, p1)) return;
    if (!__ldcg(P.any_active)) break;
    // ---- sweep B: sol += alpha s, res -= alpha As ------------------------------------------
    for (int task = t_lo + blockIdx.x; task < t_hi; task += gridDim.x) {
      const int p = task_problem(P, task, p0, p1);
      if (__ldcg(&P.state[p].phase) != 2) continue;
      const BatchProblem& pr = P.probs[p];
      const Geo g = pr.g;
      const int n = __ldcg(&P.state[p].n);
      const double alpha = __ldcg(&P.state[p].alpha);
      const double* __restrict__ sn = pr.s[n & 1];
      const int lt = task - pr.tile0;
      const int i0 = 1 + kTX * (lt % pr.ntx), j0 = 1 + kTY * (lt / pr.ntx);
      double v[2] = {0.0, 0.0};
#pragma unroll 4
      for (int e = threadIdx.x; e < kTX * kTY; e += kBatchThreads) {
        const int i = i0 + e % kTX, j = j0 + e / kTX;
        if (i > g.nx || j > g.ny) continue;
        const size_t q = g.at(i, j);
        const double w = pr.op.W[q];
        const double r = pr.res[q] - alpha * pr.As[q];
        pr.sol[q] = pr.sol[q] + alpha * sn[q];
        store_cyclic(pr.res, g, i, j, r);
        const double wd = pr.weighted ? 1.0 / (pr.op.ax[i + 1] * pr.op.by[j + 1]) : 1.0;
        v[0] += (wd * w * r) * r;
        if (w != 0.0) v[1] += r * r;
      }
      double out[2];
      block_reduce<2, -1, kBatchThreads>(v, out);
      if (threadIdx.x == 0) {
        P.part[(size_t)task * 4] = out[0];
        P.part[(size_t)task * 4 + 1] = out[1];
      }
    }
    if (!reduce_barrier(P, epoch, kSweepB, p0, p1)) return;
  }
  }  // groups
}

const void* cg_batch_kernel_ptr() { return (const void*)cg_batch_kernel; }

cudaError_t launch_cg_batch(const BatchParams& P, int grid, cudaStream_t st) {
  BatchParams Q = P;
  void* args[] = {&Q};
  return cudaLaunchCooperativeKernel((const void*)cg_batch_kernel, dim3(grid), dim3(kBatchThreads), args, 0, st);
}

}  // namespace pyomgpu
