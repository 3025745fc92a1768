// Private: the solver context behind the opaque pyomgpu_ctx handle of the C
// ABI, shared by the translation units that implement entry points
// (capi.cu, precond.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/pyomgpu.h"
#include "cg_batch.cuh"
#include "cg_pipe.cuh"
#include "cg_ref.cuh"
#include "cg_res.cuh"
#include "common.cuh"
#include "islands.h"
#include "kernels.cuh"

using pyomgpu::BatchProblem;
using pyomgpu::BatchState;
using pyomgpu::CGResParams;
using pyomgpu::CGResult;
using pyomgpu::Geo;
using pyomgpu::IslandDev;
using pyomgpu::IslandSet;
using pyomgpu::OpBuf;
using pyomgpu::OpDev;
using pyomgpu::PipeResult;
using pyomgpu::SyncCtl;

struct pyomgpu_ctx {
  int device = 0, nsm = 0;
  Geo g{};
  int nx = 0, ny = 0;
  size_t n2 = 0;  // (nx+4)*(ny+4)
  int free_surface = 0;
  double grav = 0, dt_mom = 0;
  std::vector<double> h_maskU, h_maskV;
  // device grid copies
  double *dxt = nullptr, *dxu = nullptr, *dyt = nullptr, *dyu = nullptr, *cost = nullptr, *cosu = nullptr;
  double *hur = nullptr, *hvr = nullptr, *hu = nullptr, *hv = nullptr, *mT = nullptr, *mU = nullptr, *mV = nullptr;
  OpBuf sf, sp;
  bool have_sp = false;
  // islands
  bool have_islands = false, have_psin = false, have_line_psin = false, lu_singular = false;
  IslandSet isl;
  IslandDev idev;
  std::vector<int> psin_iters;
  std::vector<double> line_psin;
  int *bnd_i = nullptr, *bnd_j = nullptr;
  int nbnd = 0;
  double* psin = nullptr;  // Fortran layout, nisle fields
  double *lu = nullptr, *line_forc = nullptr, *line_psi0 = nullptr;
  int* ipiv = nullptr;
  // CG work
  double *res = nullptr, *s0 = nullptr, *s1 = nullptr, *As = nullptr, *sol = nullptr;
  double *stage_a = nullptr, *stage_b = nullptr, *fpx = nullptr, *fpy = nullptr, *forc = nullptr, *zeros = nullptr;
  double *part = nullptr, *scal = nullptr;
  SyncCtl* ctl = nullptr;
  double* slots = nullptr;
  CGResult* d_result = nullptr;
  CGResult* h_result = nullptr;
  double* h_scal = nullptr;
  int max_blocks = 0;  // co-resident blocks of the CG kernels
  double timeout_s = 2.0;
  unsigned stall_next = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;

  // single-barrier PCG (pyomgpu_solve_rtol), allocated on first use
  struct Fast {
    bool ready = false, f32_ready = false, op32_stale = true;
    int max_blocks = 0;
    double* b = nullptr;
    double *r[2] = {}, *q[2] = {}, *w[2] = {};
    double* p = nullptr;
    OpDev<float> op32{};
    float *FX = nullptr, *FY = nullptr, *W = nullptr, *ax = nullptr, *bx = nullptr, *by = nullptr;
    float *b32 = nullptr, *x32 = nullptr, *p32 = nullptr;
    float *r32[2] = {}, *q32[2] = {}, *w32[2] = {};
    double* slots = nullptr;
    PipeResult* d_res = nullptr;
    PipeResult* h_res = nullptr;
    std::vector<void*> owned;
  } fast;

  // tile shape and grid of cg_ref_kernel chosen by pyomgpu_autotune (default 64x16, all co-resident blocks)
  struct Tune {
    bool done = false;
    int tx = 0, ty = 0, grid = 0;
    double us_per_it = 0;
  } tune;

  // on-chip-resident kernel of the streamfunction solves (cg_res.cu): piece
  // layout planned on first use, exchange buffers allocated with it
  // psin solves of streamfunction_init: the reference's stop (psin_rtol = 0), or
  // to ||res|| <= psin_rtol ||res_0||, with cell-area-weighted products if psin_weighted
  double psin_rtol = 0.0;
  int psin_weighted = 0;
  int cg_kernel = 0;  // 0 automatic, 1 tiled cg_ref_kernel, 2 resident cg_res_kernel
  struct Resident {
    bool planned = false, ok = false;
    int npx = 0, npy = 0, wmax = 0, hmax = 0, p = 0;
    size_t smem = 0;
    double *hx = nullptr, *slots = nullptr;
    unsigned tag_gen = 0;  // generation of the next solve's epoch tags (0 .. 4094)
    // FP32 instance (cg_res32_kernel, the mixed-precision correction solves)
    bool planned32 = false, ok32 = false;
    int npx32 = 0, npy32 = 0, wmax32 = 0, hmax32 = 0, p32 = 0;
    size_t smem32 = 0;
    double *hx32 = nullptr, *slots32 = nullptr;
    float* res32 = nullptr;
    // phase trace of the next resident solve (pyomgpu_resident_trace): device
    // buffer of trace_cap words, loop trips trace_it0 .. trace_it0 + trace_nit - 1
    unsigned long long* trace = nullptr;
    size_t trace_cap = 0;
    int trace_it0 = 0, trace_nit = 0;
  } resd;

  // work-queue batch (pyomgpu_congrad_streamfunction_batch and the psin
  // solves); grows to the largest batch run through this context
  struct Batch {
    int max_blocks = 0;
    double* pool = nullptr;  // per solve: padded sol, res, s0, s1, As + Fortran staging of forc, sol
    size_t cap = 0;          // doubles
    BatchProblem* d_probs = nullptr;
    BatchProblem* h_probs = nullptr;  // pinned
    BatchState* d_state = nullptr;
    BatchState* h_state = nullptr;    // pinned
    int cap_probs = 0;
    double* part = nullptr;  // 4 per task
    size_t cap_tasks = 0;
    double* d_rr = nullptr;  // 2 per solve: true residual, forcing norm
    double* h_rr = nullptr;  // pinned
    int* d_act = nullptr;    // act_n, act_prob (cap_probs), act_off (cap_probs + 1), done (cap_probs)
    int* h_act = nullptr;    // pinned: the initial act_n, act_prob, act_off
    size_t l2_bytes = 0;     // L2 size of the device
    unsigned long long* sync = nullptr;  // SyncCtl, gen
  } batch;

  // many resident solves in one launch (cg_res_multi_kernel), owned by the
  // context that runs the batch: job table, group offsets, results, error flags
  struct ResMulti {
    int cap = 0;  // jobs
    CGResParams* d_jobs = nullptr;
    CGResParams* h_jobs = nullptr;  // pinned
    int* d_idx = nullptr;           // group_base (cap + 1) then job_first (cap + 1)
    int* h_idx = nullptr;           // pinned
    CGResult* d_out = nullptr;
    CGResult* h_out = nullptr;      // pinned
    SyncCtl* d_ctl = nullptr;
    SyncCtl* h_ctl = nullptr;       // pinned
    unsigned long long* d_times = nullptr;  // 2 per job: gang assembled, piece 0 done (%globaltimer)
    unsigned long long* h_times = nullptr;  // pinned
    size_t smem_cap = 0;            // dynamic shared memory reserved for the kernel (0: not yet)
  } rmulti;
  int batch_kernel = 0;  // 0 automatic, 1 work-queue kernel, 2 resident groups
  // device time (ns) of this context's solves in the last resident batch, by
  // occurrence in that batch: the schedule's estimates for the next one
  std::vector<double> batch_ns;
  // the last resident batch run by this (owner) context, per solve in call
  // order: start and end (ms after the earliest start) and blocks used
  std::vector<double> sched_start, sched_end;
  std::vector<int> sched_blocks;
  // the solves (contexts, call order) and the schedule order of that batch: the
  // starting point of the next batch's order search when it has the same solves
  std::vector<const pyomgpu_ctx*> sched_key;
  std::vector<int> sched_order;

  ~pyomgpu_ctx() {
    for (void* p : fast.owned)
      if (p) cudaFree(p);
    if (fast.h_res) cudaFreeHost(fast.h_res);
    for (void* p : {(void*)batch.pool, (void*)batch.d_probs, (void*)batch.d_state, (void*)batch.part,
                    (void*)batch.d_rr, (void*)batch.sync})
      if (p) cudaFree(p);
    if (batch.h_probs) cudaFreeHost(batch.h_probs);
    if (batch.h_state) cudaFreeHost(batch.h_state);
    if (batch.h_rr) cudaFreeHost(batch.h_rr);
    if (batch.h_act) cudaFreeHost(batch.h_act);
    for (void* p : {(void*)rmulti.d_jobs, (void*)rmulti.d_idx, (void*)rmulti.d_out, (void*)rmulti.d_ctl,
                    (void*)rmulti.d_times})
      if (p) cudaFree(p);
    for (void* p : {(void*)rmulti.h_jobs, (void*)rmulti.h_idx, (void*)rmulti.h_out, (void*)rmulti.h_ctl,
                    (void*)rmulti.h_times})
      if (p) cudaFreeHost(p);
    for (void* p : {(void*)resd.hx, (void*)resd.slots, (void*)resd.trace, (void*)batch.d_act, (void*)resd.hx32,
                    (void*)resd.slots32, (void*)resd.res32})
      if (p) cudaFree(p);
    void* ptrs[] = {dxt, dxu, dyt, dyu, cost, cosu, hur, hvr, hu, hv, mT, mU, mV, sf.FX, sf.FY, sf.W, sf.ax, sf.bx,
                    sf.by, sp.FX, sp.FY, sp.W, sp.ax, sp.bx, sp.by, bnd_i, bnd_j, psin, lu, line_forc, line_psi0, ipiv,
                    res, s0, s1, As, sol, stage_a, stage_b, fpx, fpy, forc, zeros, part, scal, ctl, slots, d_result,
                    idev.seg_i, idev.seg_j, idev.seg_d, idev.seg_off};
    for (void* p : ptrs)
      if (p) cudaFree(p);
    if (h_result) cudaFreeHost(h_result);
    if (h_scal) cudaFreeHost(h_scal);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

// Jacobi-PCG (the reference algorithm of congrad_streamfunction with the
// relative-residual stop) on c->sol (padded, halo valid), forcing in Fortran
// layout on the device (capi.cu).
int run_pcg_from_sol(pyomgpu_ctx* c, const double* forc_dev, int max_it, double rtol, pyomgpu_solve_info* info,
                     cudaStream_t st);
