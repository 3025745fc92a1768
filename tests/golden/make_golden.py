"""Writes tests/golden/c0_oracle.npz: the oracle's results on the seeded 40x40
configuration (islands, psin, line_psin, one congrad_streamfunction solve).

The reference cannot run here (no Fortran compiler), so these fixtures pin
the oracle against later changes rather than against the reference binary.
Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from pyom2_b200 import synth  # noqa: E402


def main():
    W = synth.config0()
    M = W.M
    O = Oracle(M)
    O.streamfunction_init()
    cf = O.make_coeff_streamfunction()
    sol = np.zeros(M.shape2d, order="F")
    r = O.congrad_streamfunction(cf, W.forc, sol)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c0_oracle.npz")
    np.savez_compressed(out, forc=W.forc, boundary=M.boundary, line_dir=M.line_dir, nr_boundary=M.nr_boundary,
                        psin=M.psin, line_psin=M.line_psin, sol=sol, iterations=r["iterations"])
    print(out, r)


if __name__ == "__main__":
    main()
