// Persistent work-queue CG: many independent streamfunction solves in one
// launch, each following congrad_streamfunction's control flow
// (solve_streamfct.f90:153-327) with its own scalars.
//
// The tiles of the problems still running form one task list; every block
// walks it with a static stride.  All problems advance in lockstep through
// three kinds of sweep (init, A: direction + stencil, B: update) separated by
// grid barriers.  Every tile's arrival is counted per problem (a release
// reduction); at the end of the sweep the block that processed a problem's
// last task waits for the count, sums that problem's per-tile partials in a
// fixed order and runs its stopping logic, so every problem ends with exactly
// the iterations and status an individual solve would give; the last block
// at the barrier rebuilds the list of problems still running and releases
// the others with a generation flag.
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

__device__ __forceinline__ int ld_acquire_i32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int atom_add_acqrel_i32(int* p, int v) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Sums problem p's per-tile partials of the sweep just finished, in a fixed
// order (lane l: tiles l, l+32, ..., four loads in flight; then a shuffle
// tree), and advances its state.  Warp 0 of the block that finished the
// problem's last tile; the tiles' partials are visible through the acq_rel
// arrivals on done[p].
__device__ void reduce_problem(const BatchParams& P, int p, int kind) {
  const int lane = threadIdx.x & 31;
  const BatchProblem& pr = P.probs[p];
  const int nt = pr.ntx * pr.nty;
  const int nv = (kind == kInit) ? 4 : 2;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
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
    __stcg(&P.done[p], 0);  // ready for the next sweep (ordered before this block's barrier arrival)
  }
}

// After a tile of problem p (its partials stored by thread 0): thread 0
// counts it with a release reduction (no return value, nothing to wait for),
// which also releases those partials.
__device__ __forceinline__ void tile_finished(const BatchParams& P, int p) {
  if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(P.done + p) : "memory");
}

// End of a sweep: the block that processed a problem's last task reduces the
// problem once all its tiles have arrived (acquire poll, bounded); the
// block's warps take such problems in turn.  False on time-out.
__device__ bool reduce_own(const BatchParams& P, int kind, const int* off, const int* prb, int m) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int mine = 0;  // designated problems seen so far (every warp scans the list the same way)
  bool ok = true;
  for (int k = 0; k < m; k++) {
    if ((off[k + 1] - 1) % (int)gridDim.x != (int)blockIdx.x) continue;
    if (mine++ % (kBatchThreads / 32) != warp) continue;
    const int p = prb[k];
    const BatchProblem& pr = P.probs[p];
    const int nt = pr.ntx * pr.nty;
    if (lane == 0) {
      const unsigned long long t0 = globaltimer_ns();
      int cnt;
      unsigned spins = 0;
      while ((cnt = ld_acquire_i32(P.done + p)) < nt)
        if ((++spins & 63u) == 0u && (ld_relaxed_i32(&P.ctl->error) != 0 || globaltimer_ns() - t0 > P.timeout_ns)) {
          atomicExch(&P.ctl->error, PYOMGPU_TIMEOUT);
          break;
        }
      ok = cnt >= nt;
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    __syncwarp();
    if (!ok) break;
    reduce_problem(P, p, kind);
  }
  return ok;
}

// Grid barrier after a sweep; the last block to arrive rebuilds the list of
// problems in phase `want` (the next sweep's) and releases the others with a
// generation flag.  Every block then copies the list into shared memory
// (when it fits).  Returns false on time-out.
__device__ bool barrier_rebuild(const BatchParams& P, unsigned long long& epoch, int want, unsigned extra,
                                int* s_act_prob, int* s_act_off, int* s_actn) {
  __shared__ int s_last, s_ok;
  __syncthreads();
  epoch += 1;
  if (threadIdx.x == 0) {
    const unsigned long long old = atom_add_acqrel(&P.ctl->arrive, 1ull);
    s_last = (old + 1 == epoch * (unsigned long long)gridDim.x + extra);
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    // every problem's state of this sweep is visible (acquire side of the arrivals)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      int m = 0, off = 0;
      for (int base = 0; base < P.nprob; base += 32) {
        const int p = base + lane;
        const bool in = p < P.nprob && __ldcg(&P.state[p].phase) == want;
        const int nt = in ? P.probs[p].ntx * P.probs[p].nty : 0;
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        int sc = nt;  // inclusive scan of the tile counts
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, sc, d);
          if (lane >= d) sc += y;
        }
        if (in) {
          const int pos = m + __popc(bal & ((1u << lane) - 1u));
          __stcg(&P.act_prob[pos], p);
          __stcg(&P.act_off[pos + 1], off + sc);
        }
        m += __popc(bal);
        off += __shfl_sync(0xffffffffu, sc, 31);
      }
      __syncwarp();  // every lane's list entries before lane 0's release
      if (lane == 0) {
        __stcg(&P.act_off[0], 0);
        __stcg(P.act_n, m);
        __threadfence();
        st_release_u64(P.gen, epoch);
      }
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
  if (!s_ok) return false;
  if (s_last && threadIdx.x == 0) __threadfence();  // the list's stores before this block reads them back
  __syncthreads();
  const int m = __ldcg(P.act_n);  // at most nprob <= kBatchActMax
  for (int k = threadIdx.x; k < m; k += kBatchThreads) {
    s_act_prob[k] = __ldcg(&P.act_prob[k]);
    s_act_off[k + 1] = __ldcg(&P.act_off[k + 1]);
  }
  if (threadIdx.x == 0) {
    s_act_off[0] = 0;
    *s_actn = m;
  }
  __syncthreads();
  return true;
}

// Position of `task` in the active list: the k with off[k] <= task < off[k+1].
__device__ __forceinline__ int act_find(const int* off, int m, int task) {
  int lo = 0, hi = m - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= task)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

}  // namespace

__global__ void __launch_bounds__(kBatchThreads, 4) cg_batch_kernel(const BatchParams P) {
  __shared__ double b_s[kBoxN], b_FX[kBoxN], b_FY[kBoxN];
  __shared__ int s_act_prob[kBatchActMax], s_act_off[kBatchActMax + 1];
  __shared__ int s_actn;
  unsigned long long epoch = 0;
  // the active list of the initial sweep (every problem, nprob <= kBatchActMax), written by the host
  {
    const int m = __ldcg(P.act_n);
    for (int k = threadIdx.x; k <= m; k += kBatchThreads) {
      if (k < m) s_act_prob[k] = __ldcg(&P.act_prob[k]);
      s_act_off[k] = __ldcg(&P.act_off[k]);
    }
    if (threadIdx.x == 0) s_actn = m;
    __syncthreads();
  }
  auto list_off = [&]() -> const int* { return s_act_off; };
  auto list_prob = [&]() -> const int* { return s_act_prob; };

  // ---- init: res = forc - A sol -------------------------------------------------
  {
    const int m = s_actn;
    const int* off = list_off();
    const int* prb = list_prob();
    const int ntot = off[m];
    for (int task = blockIdx.x; task < ntot; task += gridDim.x) {
      const int k = act_find(off, m, task);
      const int p = prb[k];
      const BatchProblem& pr = P.probs[p];
      const Geo g = pr.g;
      const int lt = task - off[k];
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
        for (int c = 0; c < 4; c++) P.part[(size_t)(pr.tile0 + lt) * 4 + c] = out[c];
      tile_finished(P, p);
    }
  }
  if (!reduce_own(P, kInit, s_act_off, s_act_prob, s_actn)) return;
  if (!barrier_rebuild(P, epoch, 1, P.stall_extra, s_act_prob, s_act_off, &s_actn)) return;

  for (;;) {
    if (s_actn == 0) break;
    // ---- sweep A: s_new = Z res + bq s_old on tile + halo, As = A s_new ---------------
    {
      const int m = s_actn;
      const int* off = list_off();
      const int* prb = list_prob();
      const int ntot = off[m];
      for (int task = blockIdx.x; task < ntot; task += gridDim.x) {
        const int k = act_find(off, m, task);
        const int p = prb[k];
        const BatchProblem& pr = P.probs[p];
        const Geo g = pr.g;
        const OpDev<double> op = pr.op;
        const int n = __ldcg(&P.state[p].n);
        const double bq = __ldcg(&P.state[p].bq);
        const double* __restrict__ so = pr.s[(n + 1) & 1];
        double* __restrict__ sn = pr.s[n & 1];
        const int lt = task - off[k];
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
          const int kk = (rr + 1) * kBX + c + 1;
          const double sc = b_s[kk];
          const double a =
              op.ax[i + 1] * op.bx[j + 1] * (b_FX[kk + 1] * (b_s[kk + 1] - sc) + b_FX[kk] * (b_s[kk - 1] - sc)) +
              op.by[j + 1] * (b_FY[kk + kBX] * (b_s[kk + kBX] - sc) + b_FY[kk] * (b_s[kk - kBX] - sc));
          store_cyclic(sn, g, i, j, sc);
          pr.As[g.at(i, j)] = a;
          const double wd = pr.weighted ? 1.0 / (op.ax[i + 1] * op.by[j + 1]) : 1.0;
          v[0] += (wd * sc) * a;
          v[1] = fmax(v[1], fabs(sc));
        }
        double out[2];
        block_reduce<2, 1, kBatchThreads>(v, out);
        if (threadIdx.x == 0) {
          P.part[(size_t)(pr.tile0 + lt) * 4] = out[0];
          P.part[(size_t)(pr.tile0 + lt) * 4 + 1] = out[1];
        }
        tile_finished(P, p);
      }
    }
    if (!reduce_own(P, kSweepA, s_act_off, s_act_prob, s_actn)) return;
    if (!barrier_rebuild(P, epoch, 2, 0u, s_act_prob, s_act_off, &s_actn)) return;
    if (s_actn == 0) break;
    // ---- sweep B: sol += alpha s, res -= alpha As ------------------------------------------
    {
      const int m = s_actn;
      const int* off = list_off();
      const int* prb = list_prob();
      const int ntot = off[m];
      for (int task = blockIdx.x; task < ntot; task += gridDim.x) {
        const int k = act_find(off, m, task);
        const int p = prb[k];
        const BatchProblem& pr = P.probs[p];
        const Geo g = pr.g;
        const int n = __ldcg(&P.state[p].n);
        const double alpha = __ldcg(&P.state[p].alpha);
        const double* __restrict__ sn = pr.s[n & 1];
        const int lt = task - off[k];
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
          P.part[(size_t)(pr.tile0 + lt) * 4] = out[0];
          P.part[(size_t)(pr.tile0 + lt) * 4 + 1] = out[1];
        }
        tile_finished(P, p);
      }
    }
    if (!reduce_own(P, kSweepB, s_act_off, s_act_prob, s_actn)) return;
    if (!barrier_rebuild(P, epoch, 1, 0u, s_act_prob, s_act_off, &s_actn)) return;
  }
}

const void* cg_batch_kernel_ptr() { return (const void*)cg_batch_kernel; }

cudaError_t launch_cg_batch(const BatchParams& P, int grid, cudaStream_t st) {
  BatchParams Q = P;
  void* args[] = {&Q};
  return cudaLaunchCooperativeKernel((const void*)cg_batch_kernel, dim3(grid), dim3(kBatchThreads), args, 0, st);
}

}  // namespace pyomgpu
