"""Benchmark: ms per external-mode solve to FP64 relative residual 1e-10.

Workload (N=1): the 1440x720, 80S-80N, cyclic-in-x, 20-land-mass
streamfunction problem (seeded synthetic inputs; no data set involved).  One
step = one solve of A x = forc from a zero first guess until the FP64 true
relative residual ||forc - A x||/||forc|| over the unknowns is <= 1e-10,
through the library's C ABI (pyomgpu_solve_rtol).  Inputs are resident in HBM
for ``value``; ``e2e`` passes host buffers so the host<->device copies are in
the timed region.  L2 is flushed (256 MiB write) before every timed step.

``--impl reference`` times the oracle (the C restatement of the reference
congrad_streamfunction, same algorithm) on the host cores instead.
Multi-GPU: every rank solves its own replica (no collective on the data
path); the value is the aggregate solves/time across ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms/solve to FP64 rel. residual 1e-10: learned FCG vs plain PCG, 1 B200"
RTOL = 1e-10
BYTES_PER_POINT_ITER = {"f64": 72, "f32": 36}  # algorithmic bytes, plain PCG iteration
# DRAM bytes (read + write) per launch of the dominant kernel from one ncu capture of this
# workload (profiles/cg_ref_kernel_c1_1440x720.md), per iteration, keyed by kernel
MEASURED_TRAFFIC_PER_ITER = {"cg_ref_kernel": (1.219541e9 + 2.498041e9) / 1760}
CLOCK_Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = gpu_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={CLOCK_Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def build_workload():
    from pyom2_b200 import synth
    W = synth.config1()
    return W


def cpu_baseline(W, iterations_needed, budget_s=12.0):
    """The oracle's congrad_streamfunction (single thread, reference loop
    order) on a bounded number of iterations of the same problem."""
    from oracle.oracle import Oracle
    M = W.M.copy()
    O = Oracle(M)
    O.streamfunction_init(max_it=1, maxipp=10**6, maxq=10**6)
    cf = O.make_coeff_streamfunction()
    sol = np.zeros(M.shape2d, order="F")
    t0 = time.perf_counter()
    O.congrad_streamfunction(cf, W.forc, sol, eps=0.0, max_it=5, rtol=RTOL)
    per = (time.perf_counter() - t0) / 5
    n = max(10, min(2000, int(budget_s / max(per, 1e-6))))
    sol[...] = 0
    t0 = time.perf_counter()
    r = O.congrad_streamfunction(cf, W.forc, sol, eps=0.0, max_it=n, rtol=RTOL)
    dt = time.perf_counter() - t0
    it = r["iterations"] if r["status"] == 0 else n
    per_it = dt / max(1, min(it, n))
    return {"value": per_it * iterations_needed * 1e3, "unit": "ms/solve", "cores": 1, "kind": "port",
            "sample": f"{min(it, n)} PCG iterations of the 1440x720 solve timed ({dt:.1f} s), "
                      f"x {iterations_needed} iterations per solve"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    W = build_workload()
    from oracle.oracle import Oracle
    M = W.M.copy()
    O = Oracle(M)
    O.streamfunction_init(max_it=1, maxipp=10**6, maxq=10**6)
    cf = O.make_coeff_streamfunction()
    # the reference algorithm's own iteration count to the residual target
    sol = np.zeros(M.shape2d, order="F")
    r = O.congrad_streamfunction(cf, W.forc, sol, eps=0.0, max_it=100000, rtol=RTOL)
    need = r["iterations"]
    per = []
    sample = 60
    for k in range(args.warmup + args.steps):
        sol[...] = 0
        t0 = time.perf_counter()
        O.congrad_streamfunction(cf, W.forc, sol, eps=0.0, max_it=sample, rtol=RTOL)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            per.append(dt / sample)
    ms = statistics.median(per) * need * 1e3
    line = {"metric": METRIC, "value": ms, "unit": "ms/solve", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "c1_1440x720_20isl_cyclic", "rtol": RTOL, "method": "Jacobi-PCG (reference)"},
            "impl": "reference",
            "cpu_baseline": {"value": ms, "unit": "ms/solve", "cores": 1, "kind": "port",
                             "sample": f"{sample} iterations per step x {need} iterations per solve"},
            "e2e": {"value": ms, "unit": "ms/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from pyom2_b200 import _abi
    from pyom2_b200.external import ExternalMode, _ptr

    W = build_workload()
    M = W.M
    E = ExternalMode(M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6)
    prec = _abi.PREC_F64 if args.precision == "f64" else _abi.PREC_F32
    dev = torch.device("cuda", local)
    forc_d = torch.from_numpy(np.ascontiguousarray(W.forc.T)).to(dev).T
    sol_d = torch.zeros(tuple(reversed(M.shape2d)), dtype=torch.float64, device=dev).T
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    L = _abi.load()

    def solve_device():
        sol_d.zero_()
        info = _abi.SolveInfo()
        rc = L.pyomgpu_solve_rtol(E._ctx, _ptr(forc_d), _ptr(sol_d), RTOL, prec, 1000000, C.byref(info),
                                  C.c_void_p(stream.cuda_stream))
        _abi.check(rc)
        return info

    for _ in range(args.warmup):
        solve_device()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    times, kern, iters, relres = [], [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info = solve_device()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            kern.append(info.device_ms)
            iters.append(info.iterations)
            relres.append(info.rel_residual)
    torch.cuda.synchronize()
    total_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = total_ms / (args.steps * world)  # aggregate: all ranks' solves over the max rank time

    # end to end through the C ABI with host buffers (copies inside the timed region)
    forc_h = np.asfortranarray(W.forc)
    sol_h = np.zeros(M.shape2d, order="F")
    e2e = []
    for k in range(args.warmup + max(3, args.steps // 2)):
        sol_h[...] = 0
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = _abi.SolveInfo()
        rc = L.pyomgpu_solve_rtol(E._ctx, _ptr(forc_h), _ptr(sol_h), RTOL, prec, 1000000, C.byref(info),
                                  C.c_void_p(stream.cuda_stream))
        _abi.check(rc)
        dt = (time.perf_counter() - t0) * 1e3
        if k >= args.warmup:
            e2e.append(dt)
    n2 = M.shape2d[0] * M.shape2d[1]

    N = M.nx * M.ny
    it_med = int(statistics.median(iters))
    kern_med = statistics.median(kern)
    alg_bytes = BYTES_PER_POINT_ITER[args.precision] * N * it_med
    achieved = alg_bytes / (kern_med * 1e-3) / 1e9
    peak, peak_kind = peaks()
    out = {
        "metric": METRIC, "value": value, "unit": "ms/solve", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {"workload": "c1_1440x720_20isl_cyclic", "nx": M.nx, "ny": M.ny, "nisle": int(M.nisle),
                   "rtol": RTOL, "method": f"Jacobi-PCG {args.precision} (reference algorithm, persistent kernel)",
                   "iterations": it_med, "max_rel_residual": max(relres), "l2": "flushed (256 MiB write) per step",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (MEASURED_TRAFFIC_PER_ITER["cg_ref_kernel"] * it_med
                                 if args.precision == "f64" else None),
                     "algorithmic_bytes": alg_bytes, "peak_kind": peak_kind, "kernel": "cg_ref_kernel",
                     "kernel_ms": kern_med, "bytes_per_point_iter": BYTES_PER_POINT_ITER[args.precision]},
        "e2e": {"value": statistics.median(e2e), "unit": "ms/solve", "h2d_bytes_per_step": 2 * n2 * 8,
                "d2h_bytes_per_step": n2 * 8},
        "gpu_launches": 6 * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(W, it_med)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
