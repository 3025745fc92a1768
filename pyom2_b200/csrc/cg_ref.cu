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
//   sweep A: per tile, TMA loads of res, W, s_old, FX, FY (tile + halo) into
//            shared memory; s_new = W1*res + (beta/beta_old)*s_old on the tile
//            and its one-cell halo (recomputed locally, so no barrier is needed
//            before the stencil); As = A s_new; partials (s,As), max|s|
//   sweep B: per point, sol += alpha*s_new; res -= alpha*As; partial
//            beta_next = (W1 res, res)
//
// The search direction is double-buffered (s_old is read by neighbouring
// tiles while s_new is written).  Cyclic halos are written by the owner of the
// source point (setcyclic_xy, parallel_none.f90:188-211).
#include <math.h>

#include "cg_ref.cuh"

namespace pyomgpu {

__device__ __forceinline__ void tile_origin(const CGRefParams& P, int t, int& i0, int& j0) {
  i0 = 1 + P.tx * (t % P.ntx);
  j0 = 1 + P.ty * (t / P.ntx);
}

template <bool SP>
__global__ void __launch_bounds__(kCGThreads, 3) cg_ref_kernel(const __grid_constant__ CGRefParams P) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int TX = P.tx, TY = P.ty, BX = TX + 4, BY = TY + 2;
  constexpr int kCGWarps = kCGThreads / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t tb = cg_box_bytes(TX, TY);
  double* tres = reinterpret_cast<double*>(smem);
  double* tW = reinterpret_cast<double*>(smem + tb);
  double* ts = reinterpret_cast<double*>(smem + 2 * tb);
  double* tFX = reinterpret_cast<double*>(smem + 3 * tb);
  double* tFY = reinterpret_cast<double*>(smem + 4 * tb);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 5 * tb);

  const Geo g = P.g;
  const OpDev<double> op = P.op;
  const unsigned nb = gridDim.x;
  const int ntiles = P.ntx * P.nty;
  unsigned long long epoch = 0;
  uint32_t phase = 0;
  double* __restrict__ res = P.res;
  double* __restrict__ As = P.As;
  double* __restrict__ sol = P.sol;
  const double* __restrict__ Wf = op.W;
  const double F_1EM10 = (double)1.e-10f;  // solve_streamfct.f90:262, a default-real literal

  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();

  // ------------------------------------------------------------------ init
  // res = forc - A sol (interior), solve_streamfct.f90:196-201 / solve_pressure.f90:163-168
  {
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // beta, bb, rr, zresmax
    for (int t = blockIdx.x; t < ntiles; t += nb) {
      int i0, j0;
      tile_origin(P, t, i0, j0);
      for (int e = threadIdx.x; e < TX * TY; e += kCGThreads) {
        const int i = i0 + e % TX, j = j0 + e / TX;
        if (i > g.nx || j > g.ny) continue;
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
  grid_collect<4, 3, kCGThreads>(P.slots, 4, nb, red);
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
      double* __restrict__ sn = P.s[n & 1];
      const CUtensorMap* map_so = &P.map_s[(n + 1) & 1];
      double acc_dot = 0.0, acc_max = 0.0;
      for (int t = blockIdx.x; t < ntiles; t += nb) {
        int i0, j0;
        tile_origin(P, t, i0, j0);
        __syncthreads();  // the previous tile's shared-memory reads are done
        if (threadIdx.x == 0) {
          fence_proxy_async_smem();
          fence_proxy_async_global();
          mbar_arrive_expect_tx(bar, 5u * (unsigned)(BX * BY) * 8u);
          const int ex = i0 + 1, ey = j0;  // padded element column of Fortran i0-2, row of j0-1
          tma_load_2d(tres, &P.map_res, ex, ey, bar);
          tma_load_2d(tW, &P.map_W, ex, ey, bar);
          tma_load_2d(ts, map_so, ex, ey, bar);
          tma_load_2d(tFX, &P.map_FX, ex, ey, bar);
          tma_load_2d(tFY, &P.map_FY, ex, ey, bar);
        }
        const bool ok = __syncthreads_and(mbar_wait_bounded(bar, phase, P.timeout_ns));
        phase ^= 1u;
        if (!ok) {
          if (threadIdx.x == 0) atomicExch(&P.ctl->error, PYOMGPU_TIMEOUT);
          return;
        }
        // direction on the tile and its one-cell halo: box columns 1..BX-2, all rows
        // (rows to warps, columns to lanes: no division by the run-time tile width)
        for (int rr = warp; rr < BY; rr += kCGWarps)
          for (int k = rr * BX + 1 + lane; k < rr * BX + BX - 1; k += 32) {
            const double w1 = SP ? 1.0 : tW[k];
            ts[k] = w1 * tres[k] + bq * ts[k];
          }
        __syncthreads();
        for (int r = warp; r < TY; r += kCGWarps)
          for (int c = lane; c < TX; c += 32) {
          const int i = i0 + c, j = j0 + r;
          if (i > g.nx || j > g.ny) continue;
          const int k = (r + 1) * BX + c + 2;
          const double sc = ts[k];
          double a = op.ax[i + 1] * op.bx[j + 1] * (tFX[k + 1] * (ts[k + 1] - sc) + tFX[k] * (ts[k - 1] - sc)) +
                     op.by[j + 1] * (tFY[k + BX] * (ts[k + BX] - sc) + tFY[k] * (ts[k - BX] - sc));
          const double w = tW[k];
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
    double sAs, smax;
    {
      double r2[2];
      grid_collect<2, 1, kCGThreads>(P.slots + (size_t)((ep_a & 1) * nb) * 4, 4, nb, r2);
      sAs = r2[0];
      smax = r2[1];
    }

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
      for (int t = blockIdx.x; t < ntiles; t += nb) {
        int i0, j0;
        tile_origin(P, t, i0, j0);
        for (int r = warp; r < TY; r += kCGWarps)
          for (int c = lane; c < TX; c += 32) {
          const int i = i0 + c, j = j0 + r;
          if (i > g.nx || j > g.ny) continue;
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
      double r2[2];
      grid_collect<2, -1, kCGThreads>(P.slots + (size_t)((ep_b & 1) * nb) * 4, 4, nb, r2);
      beta_next = r2[0];
      rr_next = r2[1];
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

template __global__ void cg_ref_kernel<false>(const __grid_constant__ CGRefParams P);
template __global__ void cg_ref_kernel<true>(const __grid_constant__ CGRefParams P);

const void* cg_ref_kernel_ptr(bool sp) {
  return sp ? (const void*)cg_ref_kernel<true> : (const void*)cg_ref_kernel<false>;
}

// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

namespace {
EncodeTiledFn tiled_encoder() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return nullptr;
    fn = (EncodeTiledFn)p;
  }
  return fn;
}
}  // namespace

int encode_tile_map(CUtensorMap* map, const double* base, const Geo& g, int box_x, int box_y) {
  EncodeTiledFn fn = tiled_encoder();
  if (!fn) return -1;
  const cuuint64_t dims[2] = {(cuuint64_t)g.pitch, (cuuint64_t)(g.ny + 2 * kOnx)};
  const cuuint64_t strides[1] = {(cuuint64_t)g.pitch * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)box_y};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (int)r;
}

int encode_map(CUtensorMap* map, CUtensorMapDataType dtype, int rank, const void* base, const uint64_t* dims,
               const uint64_t* strides_bytes, const uint32_t* box) {
  EncodeTiledFn fn = tiled_encoder();
  if (!fn || rank < 1 || rank > 5) return -1;
  cuuint64_t d[5], s[4];
  cuuint32_t b[5], es[5];
  for (int k = 0; k < rank; k++) {
    d[k] = dims[k];
    b[k] = box[k];
    es[k] = 1;
    if (k < rank - 1) s[k] = strides_bytes[k];
  }
  CUresult r = fn(map, dtype, (cuuint32_t)rank, (void*)base, d, s, b, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (int)r;
}

}  // namespace pyomgpu
