"""Writes tests/golden/c1_oracle.npz: the oracle's congrad_streamfunction on
the seeded 1440x720 workload (synth.config1: 80S-80N, cyclic in x, 20 land
masses), the configuration the benchmark times.

Two solves from a zero first guess, both with the serial oracle
(oracle/pyom_oracle.c, the reference's loop order):

* the reference stop: congr_epsilon = 1e-12 (as a default real) and
  congr_max_iterations = 1000 (main_module.f90:189-190).  On this grid the
  reference's stopping estimate does not fire within 1000 iterations, so the
  solve ends with its max-iterations status after iteration 1000
  (solve_streamfct.f90:303-304): the fixture holds that iterate;
* a tight solve (eps = 0, stop at the FP64 relative residual 1e-14): the
  reference solution that every method's error is measured against.

Stored: iteration counts and statuses, the interior L2 norms and a strided
sample (every 24th column, every 12th row of the interior) of both
solutions, plus the oracle's iteration count to the benchmark's 2e-11
residual.  The GPU tests recompute both solves with the oracle at run time,
check them against this file (so the oracle is pinned across machines) and
compare the GPU solutions with the full fields.

Run: python tests/golden/make_c1_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from pyom2_b200 import synth  # noqa: E402

SAMPLE = (slice(2, -2, 24), slice(2, -2, 12))
RTOL_TIGHT = 1e-14
RTOL_BENCH = 2e-11


def oracle_solves(W):
    """(reference-stop result, its solution, tight result, tight solution,
    bench-rtol result) of the serial oracle on workload W."""
    M = W.M.copy()
    O = Oracle(M)
    O.streamfunction_init(max_it=1, maxipp=10**6, maxq=10**6)  # island lists only; psin is not used here
    cf = O.make_coeff_streamfunction()
    ref = np.zeros(M.shape2d, order="F")
    r_ref = O.congrad_streamfunction(cf, W.forc, ref)
    tight = np.zeros(M.shape2d, order="F")
    r_tight = O.congrad_streamfunction(cf, W.forc, tight, eps=0.0, max_it=10**6, rtol=RTOL_TIGHT)
    tmp = np.zeros(M.shape2d, order="F")
    r_bench = O.congrad_streamfunction(cf, W.forc, tmp, eps=0.0, max_it=10**6, rtol=RTOL_BENCH)
    return r_ref, ref, r_tight, tight, r_bench


def norm_interior(a):
    return float(np.linalg.norm(a[2:-2, 2:-2]))


def main():
    W = synth.config1()
    r_ref, ref, r_tight, tight, r_bench = oracle_solves(W)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c1_oracle.npz")
    np.savez_compressed(out, ref_iterations=r_ref["iterations"], ref_status=r_ref["status"],
                        ref_norm=norm_interior(ref), ref_sample=ref[SAMPLE],
                        tight_iterations=r_tight["iterations"], tight_status=r_tight["status"],
                        tight_norm=norm_interior(tight), tight_sample=tight[SAMPLE],
                        bench_iterations=r_bench["iterations"], rtol_tight=RTOL_TIGHT, rtol_bench=RTOL_BENCH)
    print(out, r_ref, r_tight, r_bench)


if __name__ == "__main__":
    main()
