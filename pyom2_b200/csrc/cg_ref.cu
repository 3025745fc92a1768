// Persistent, grid-synchronised conjugate-gradient kernels that reproduce the
// control flow of pyOM2's two external-mode solvers:
//
//   SP = false: congrad_streamfunction (solve_streamfct.f90:153-327), Jacobi
//               preconditioner Z with Z = 0 on island perimeters (Dirichlet),
//               Euclidean products dot_sfc/absmax_sfc (:331-362).
//   SP = true:  congrad_surf_press (solve_pressure.f90:137-249), no
//               preconditioner, products weighted by maskT(:,:,nz)
//               (dot_sfp/absmax_sfp, :277-311).
//
// One launch runs the whole solve.  Each iteration is two sweeps separated by
// grid barriers that carry the reductions (the reference's global_sum /
// global_max, parallel_mpi.f90:232-277):
//
//   sweep A: s_new = W1*res + (beta/beta_old)*s_old on the strip plus a one-cell
//            halo (recomputed locally, so no extra barrier is needed before the
//            stencil), As = A s_new; partials (s,As), max|s|
//   sweep B: sol += alpha*s_new; res -= alpha*As; partial beta_next = (W1 res, res)
//
// The search direction is double-buffered (s_old is read by neighbouring
// strips while s_new is written).  Cyclic halos are written by the owner of
// the source point (setcyclic_xy, parallel_none.f90:188-211).
//
// Work decomposition: a warp owns a strip of 32 consecutive columns x R rows;
// lane L owns column x0+1+L and walks the rows with a 3-row register window.
// x-neighbours come from warp shuffles, the two columns outside the strip from
// one extra predicated load per row.
#include <math.h>

#include "cg_ref.cuh"

namespace pyomgpu {

constexpr unsigned kFull = 0xffffffffu;

template <bool SP>
__device__ __forceinline__ void strip_coords(const CGRefParams& P, int s, int& x0, int& y0, int& jend) {
  const int sx = s % P.SX, sy = s / P.SX;
  x0 = 32 * sx;
  y0 = P.R * sy;
  jend = min(y0 + P.R, P.g.ny);
}

template <bool SP>
__global__ void __launch_bounds__(kCGThreads, 2) cg_ref_kernel(const CGRefParams P) {
  const Geo g = P.g;
  const OpDev<double> op = P.op;
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (kCGThreads / 32) + (threadIdx.x >> 5);
  const int nwarps = gridDim.x * (kCGThreads / 32);
  const int nstrips = P.SX * P.SY;
  const unsigned nb = gridDim.x;
  unsigned long long epoch = 0;
  double* __restrict__ res = P.res;
  double* __restrict__ As = P.As;
  double* __restrict__ sol = P.sol;
  const double* __restrict__ Wf = op.W;
  const double F_1EM10 = (double)1.e-10f;  // solve_streamfct.f90:262, a default-real literal

  // ------------------------------------------------------------------ init
  // res = forc - A sol (interior), solve_streamfct.f90:196-201 / solve_pressure.f90:163-168
  {
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // beta, bb, rr, zresmax
    for (int s = gw; s < nstrips; s += nwarps) {
      int x0, y0, jend;
      strip_coords<SP>(P, s, x0, y0, jend);
      const int i = x0 + 1 + lane;
      if (i > g.nx) continue;
      for (int j = y0 + 1; j <= jend; j++) {
        const double f = P.forc[fidx(g.nx, i, j)];
        const double r = f - apply_point(op, g, sol, i, j);
        store_cyclic(res, g, i, j, r);
        const double w = Wf[g.at(i, j)];
        if (SP) {
          v[0] += r * r * w;
          v[1] += f * f * w;
          v[2] += r * r * w;
        } else {
          const double zr = w * r;
          v[0] += zr * r;
          if (w != 0.0) {
            v[1] += f * f;
            v[2] += r * r;
          }
          v[3] = fmax(v[3], fabs(zr));
        }
      }
    }
    double out[4];
    block_reduce<4, 3, kCGThreads>(v, out);
    if (threadIdx.x == 0) {
      double* slot = P.slots + (size_t)blockIdx.x * 4;
      for (int k = 0; k < 4; k++) slot[k] = out[k];
    }
  }
  if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns, P.stall_extra)) return;
  double red[4];
  grid_allreduce<4, 3>(P.slots, nb, red);
  double beta = red[0];
  const double bb = red[1];
  double rr = red[2];
  const double zresmax = red[3];
  const double rtol2bb = P.rtol * P.rtol * bb;

  const double eps = P.eps;
  const int max_it = P.max_it;
  double betam1 = 1.0, betamin = 0.0, step1 = 0.0, est = 0.0, bq = 0.0;
  double alpha_prev = 0.0, rr_prev = rr;
  int n = 0, status = PYOMGPU_OK, converged = 0;

  if (!SP) {
    if (100.0 * zresmax < eps) {  // solve_streamfct.f90:210-213
      est = 100.0 * zresmax;
      n = 0;
      goto done_ok;
    }
  } else {
    if (beta == 0.0) {  // solve_pressure.f90:174-177
      n = 0;
      goto done_ok;
    }
    if (max_it < 1) {
      n = 1;
      status = PYOMGPU_MAXITER;
      goto done_err;
    }
  }

  for (n = 1;; n++) {
    if (!SP) {
      if (n > max_it) {  // solve_streamfct.f90:303-304
        status = PYOMGPU_MAXITER;
        goto done_err;
      }
      if (beta != beta) {  // early NaN stop (the reference runs on and halts at the end)
        est = beta;
        status = PYOMGPU_NAN;
        goto done_err;
      }
      if (n == 1) {  // :232-240
        betamin = fabs(beta);
      } else if (n > 2) {
        betamin = fmin(betamin, fabs(beta));
        if (fabs(beta) > 100.0 * betamin) {
          status = PYOMGPU_DIVERGED;
          goto done_err;
        }
      }
      bq = beta / betam1;  // :244
    }
    // -------------------------------------------------------------- sweep A
    {
      const double* __restrict__ so = P.s[(n + 1) & 1];
      double* __restrict__ sn = P.s[n & 1];
      double acc_dot = 0.0, acc_max = 0.0;
      for (int s = gw; s < nstrips; s += nwarps) {
        int x0, y0, jend;
        strip_coords<SP>(P, s, x0, y0, jend);
        const int i = x0 + 1 + lane;
        const bool own = i <= g.nx;
        const bool valid = i <= g.nx + 1;
        const int ie = (lane == 0) ? x0 : x0 + 33;
        const bool edge = (lane == 0) || (lane == 31 && x0 + 33 <= g.nx + 1);
        const double axi = valid ? op.ax[i + 1] : 0.0;
        auto dirv = [&](int ii, int jj) -> double {
          const size_t q = g.at(ii, jj);
          const double r = res[q];
          const double w1 = SP ? 1.0 : Wf[q];
          return w1 * r + bq * so[q];
        };
        double sm = valid ? dirv(i, y0) : 0.0;
        double sc = valid ? dirv(i, y0 + 1) : 0.0;
        double fys = valid ? op.FY[g.at(i, y0 + 1)] : 0.0;
        for (int j = y0 + 1; j <= jend; j++) {
          const double snx = valid ? dirv(i, j + 1) : 0.0;
          const double sedge = edge ? dirv(ie, j) : 0.0;
          const double fxw = valid ? op.FX[g.at(i, j)] : 0.0;
          const double fxedge = (lane == 31 && edge) ? op.FX[g.at(x0 + 33, j)] : 0.0;
          const double fyn = valid ? op.FY[g.at(i, j + 1)] : 0.0;
          double sW = __shfl_up_sync(kFull, sc, 1);
          double sE = __shfl_down_sync(kFull, sc, 1);
          double fxe = __shfl_down_sync(kFull, fxw, 1);
          if (lane == 0) sW = sedge;
          if (lane == 31) {
            sE = sedge;
            fxe = fxedge;
          }
          if (own) {
            const double sxx = axi * op.bx[j + 1];
            const double syy = op.by[j + 1];
            double a = sxx * (fxe * (sE - sc) + fxw * (sW - sc)) + syy * (fyn * (snx - sc) + fys * (sm - sc));
            const double w = Wf[g.at(i, j)];
            if (SP) a += op.dcoef * w * sc;
            store_cyclic(sn, g, i, j, sc);
            As[g.at(i, j)] = a;
            if (SP) {
              acc_dot += sc * a * w;
              acc_max = fmax(acc_max, fabs(sc * w));
            } else {
              acc_dot += sc * a;
              acc_max = fmax(acc_max, fabs(sc));
            }
          }
          sm = sc;
          sc = snx;
          fys = fyn;
        }
      }
      double v[2] = {acc_dot, acc_max}, out[2];
      block_reduce<2, 1, kCGThreads>(v, out);
      if (threadIdx.x == 0) {
        double* slot = P.slots + (size_t)((epoch & 1) * nb + blockIdx.x) * 4;
        slot[0] = out[0];
        slot[1] = out[1];
      }
    }
    const unsigned long long ep_a = epoch;
    if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns)) return;
    double ra[4];
    {
      double r2[2];
      // slots written before this barrier live in parity (ep_a & 1)
      const double* sl = P.slots + (size_t)((ep_a & 1) * nb) * 4;
      __shared__ double shr[2];
      if (threadIdx.x < 32) {
        double d = 0.0, m = 0.0;
        for (unsigned b = threadIdx.x; b < nb; b += 32) {
          d += __ldcg(sl + (size_t)b * 4);
          m = fmax(m, __ldcg(sl + (size_t)b * 4 + 1));
        }
        d = warp_sum(d);
        m = warp_max(m);
        if (threadIdx.x == 0) {
          shr[0] = d;
          shr[1] = m;
        }
      }
      __syncthreads();
      r2[0] = shr[0];
      r2[1] = shr[1];
      __syncthreads();
      ra[0] = r2[0];
      ra[1] = r2[1];
    }
    const double sAs = ra[0], smax = ra[1];

    bool stop_after = false;
    if (SP) {
      if (n > 1) {  // convergence test of iteration n-1 needs max|p| of the new p (solve_pressure.f90:209-226)
        const int m = n - 1;
        const double step = fabs(alpha_prev) * smax;
        if (m == 1) {
          step1 = step;
          est = step;
          if (step < eps) {
            n = m;
            goto done_ok;
          }
        } else if (step < eps) {
          const double rate = exp(log(step / step1) / (double)(m - 1));
          est = step * rate / (1.0 - rate);
          if (est < eps) {
            n = m;
            goto done_ok;
          }
        }
        if (est != est) {
          n = m;
          status = PYOMGPU_NAN;
          goto done_err;
        }
        if (P.rtol > 0.0 && (bb > 0.0 ? rr_prev <= rtol2bb : rr_prev == 0.0)) {
          est = sqrt(rr_prev);
          n = m;
          goto done_ok;
        }
        if (m >= max_it) {  // solve_pressure.f90:228-229
          n = max_it + 1;
          status = PYOMGPU_MAXITER;
          goto done_err;
        }
      }
      if (sAs == 0.0) goto done_ok;  // solve_pressure.f90:185
    } else {
      if (fabs(sAs) < fabs(beta) * F_1EM10) {  // solve_streamfct.f90:262-266
        est = 100.0 * smax;
        goto done_ok;
      }
    }
    const double alpha = beta / sAs;
    if (!SP) {  // solve_streamfct.f90:283-297 (decided now, applied after the update)
      const double step = fabs(alpha) * smax;
      if (n == 1) {
        step1 = step;
        est = step;
        stop_after = step < eps;
      } else if (step < eps) {
        const double rate = exp(log(step / step1) / (double)(n - 1));
        est = step * rate / (1.0 - rate);
        stop_after = est < eps;
      }
    }
    // -------------------------------------------------------------- sweep B
    {
      const double* __restrict__ sn = P.s[n & 1];
      double acc_b = 0.0, acc_r = 0.0;
      for (int s = gw; s < nstrips; s += nwarps) {
        int x0, y0, jend;
        strip_coords<SP>(P, s, x0, y0, jend);
        const int i = x0 + 1 + lane;
        if (i > g.nx) continue;
        for (int j = y0 + 1; j <= jend; j++) {
          const size_t q = g.at(i, j);
          const double sc = sn[q];
          const double w = Wf[q];
          const double r = res[q] - alpha * As[q];
          if (SP) {
            // psi(:,:,taup1) += alpha*p over the whole array (solve_pressure.f90:187)
            add_cyclic(sol, g, i, j, alpha * sc);
            acc_b += r * r * w;
            acc_r += r * r * w;
          } else {
            sol[q] = sol[q] + alpha * sc;  // solve_streamfct.f90:278
            const double zr = w * r;
            acc_b += zr * r;
            if (w != 0.0) acc_r += r * r;
          }
          store_cyclic(res, g, i, j, r);
        }
      }
      if (!SP && stop_after) goto done_ok;
      double v[2] = {acc_b, acc_r}, out[2];
      block_reduce<2, -1, kCGThreads>(v, out);
      if (threadIdx.x == 0) {
        double* slot = P.slots + (size_t)((epoch & 1) * nb + blockIdx.x) * 4;
        slot[0] = out[0];
        slot[1] = out[1];
      }
    }
    const unsigned long long ep_b = epoch;
    if (!grid_sync(P.ctl, nb, epoch, P.timeout_ns)) return;
    double beta_next, rr_next;
    {
      const double* sl = P.slots + (size_t)((ep_b & 1) * nb) * 4;
      __shared__ double shb[2];
      if (threadIdx.x < 32) {
        double d = 0.0, m = 0.0;
        for (unsigned b = threadIdx.x; b < nb; b += 32) {
          d += __ldcg(sl + (size_t)b * 4);
          m += __ldcg(sl + (size_t)b * 4 + 1);
        }
        d = warp_sum(d);
        m = warp_sum(m);
        if (threadIdx.x == 0) {
          shb[0] = d;
          shb[1] = m;
        }
      }
      __syncthreads();
      beta_next = shb[0];
      rr_next = shb[1];
      __syncthreads();
    }
    if (SP) {
      const double rsnew = beta_next;
      bq = rsnew / beta;  // p = res + rsnew/rsold*p (solve_pressure.f90:190)
      beta = rsnew;
      if (n == 1) {  // :197-205
        betamin = fabs(rsnew);
      } else if (n > 2) {
        betamin = fmin(betamin, fabs(rsnew));
        if (fabs(rsnew) > 100.0 * betamin) {
          status = PYOMGPU_DIVERGED;
          goto done_err;
        }
      }
      alpha_prev = alpha;
      rr_prev = rr_next;
    } else {
      if (P.rtol > 0.0 && (bb > 0.0 ? rr_next <= rtol2bb : rr_next == 0.0)) {
        est = sqrt(rr_next);
        goto done_ok;
      }
      betam1 = beta;
      beta = beta_next;
    }
    rr = rr_next;
  }

done_ok:
  converged = 1;
  status = PYOMGPU_OK;
  goto done;
done_err:
  converged = 0;
  if (est != est) status = PYOMGPU_NAN;
done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.out->iterations = n;
    P.out->converged = converged;
    P.out->status = status;
    P.out->est = est;
  }
}

template __global__ void cg_ref_kernel<false>(const CGRefParams P);
template __global__ void cg_ref_kernel<true>(const CGRefParams P);

const void* cg_ref_kernel_ptr(bool sp) {
  return sp ? (const void*)cg_ref_kernel<true> : (const void*)cg_ref_kernel<false>;
}

}  // namespace pyomgpu
