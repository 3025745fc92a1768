"""Train the learned preconditioner on the 1440x720 grid family on the GPU.

    python -m pyom2_b200.train_precond --out weights.npz [--steps N] [--grids 2001,2002,...]

Grids come from the 1440x720 global recipe (cyclic x, about 30 % land, 20
land masses) with the given seeds; the grid solved by the benchmark (seed
1001) is never a training grid.  Each grid gets seeded right-hand-side bases
(smooth curl forcing with 2-24 cell correlation lengths); training pairs
(residual, error) are produced on the fly by the plain Jacobi-PCG solver
(learned.generate_and_train).  One network is moved round-robin over the
grids in blocks of steps, keeping its Adam state.
"""
from __future__ import annotations

import argparse
import time
import warnings

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--block", type=int, default=250, help="steps per grid before moving on")
    ap.add_argument("--grids", default="2001,2002,2003,2004")
    ap.add_argument("--nx", type=int, default=1440)
    ap.add_argument("--ny", type=int, default=720)
    ap.add_argument("--basis", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--init", default=None, help="start from these parameters (npz)")
    a = ap.parse_args(argv)

    from . import learned, synth
    from .external import ExternalMode

    t0 = time.time()
    seeds = [int(s) for s in a.grids.split(",") if s]
    grids = []
    for s in seeds:
        W = synth._global_like(a.nx, a.ny, -80.0, 80.0, s, n_land_masses=20, name=f"train_{s}")
        E = ExternalMode(W.M)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            E.streamfunction_init(maxipp=10**6, maxq=10**6)
        grids.append((W, E, learned.rhs_basis(W, a.basis, seed=10 * s + 1)))
        print(f"grid {s}: nisle {W.M.nisle} ({time.time() - t0:.1f} s)", flush=True)
    params = learned.load_params(a.init) if a.init else learned.init_params(a.seed)
    pc = learned.LearnedPreconditioner(grids[0][1], params=params, training=True)
    losses = []
    done, k = 0, 0
    while done < a.steps:
        W, E, basis = grids[k % len(grids)]
        pc.rebind(E)
        n = min(a.block, a.steps - done)
        lr_a = a.lr * (a.lr_final / a.lr) ** (done / max(1, a.steps))
        lr_b = a.lr * (a.lr_final / a.lr) ** ((done + n) / max(1, a.steps))
        ls = learned.generate_and_train(pc, W, E, basis, n, lr_a, seed=a.seed * 1000 + k, lr_final=lr_b)
        losses += ls
        done += n
        k += 1
        print(f"steps {done}: loss(block) {np.mean(ls):.4f} last50 {np.mean(ls[-50:]):.4f} "
              f"({time.time() - t0:.1f} s)", flush=True)
    np.savez(a.out, params=pc.get_params(), losses=np.asarray(losses, dtype=np.float32),
             grids=np.asarray(seeds), nx=a.nx, ny=a.ny, steps=a.steps)
    print(f"saved {a.out} after {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main()
