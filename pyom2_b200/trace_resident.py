"""Phase timing of the on-chip-resident solve kernel (diagnostics).

Runs one FP64 solve of the 1440x720 workload (or another grid of
``synth``) in the traced instantiation of the resident kernel
(pyomgpu_resident_trace: the same arithmetic, %globaltimer stamps at every
phase boundary of a window of iterations in every block) and prints, per
phase, the median and 90th percentile over blocks and iterations of the time
spent since the previous stamp, the skew between blocks at the reductions,
and the iteration period.

    python -m pyom2_b200.trace_resident [--it0 400] [--nit 64] [--json out.json]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import warnings

import numpy as np

PHASES = ["sweepA start", "direction in smem", "stencil+partials", "S1(A)", "S2(A)", "residual+stage",
          "records written", "S1(B)", "solution update", "S2(B)+halo", "ctl S1(A)", "ctl publish(A)",
          "ctl acquire(A)", "ctl step(A)", "ctl S1(B)", "ctl publish(B)", "ctl acquire(B)", "ctl step(B)"]
NPH = len(PHASES)

# (label, from phase, to phase) intervals of one iteration
INTERVALS = [
    ("direction + halo direction", 0, 1),
    ("stencil, (s,As), max|s| partials", 1, 2),
    ("workers: wait S1(A)", 2, 3),
    ("workers: wait S2(A) (reduction A)", 3, 4),
    ("residual update + staging", 4, 5),
    ("exchange records out", 5, 6),
    ("workers: wait S1(B)", 6, 7),
    ("solution update", 7, 8),
    ("workers: wait S2(B) (reduction B + halo)", 8, 9),
    ("ctl: publish A", 10, 11),
    ("ctl: acquire all slots A", 11, 12),
    ("ctl: control step A", 12, 13),
    ("ctl: publish B", 14, 15),
    ("ctl: acquire all slots B", 15, 16),
    ("ctl: control step B", 16, 17),
]


def run(W, it0, nit, rtol=2e-11):
    import torch

    from pyom2_b200 import _abi
    from pyom2_b200.external import ExternalMode, _ptr, _stream

    E = ExternalMode(W.M)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(maxipp=10**6, maxq=10**6)
    f = torch.from_numpy(np.ascontiguousarray(W.forc.T)).cuda().T
    x = torch.zeros_like(f.T).T
    L = _abi.load()
    lay = E.resident_layout()
    nb = lay[0] * lay[1]
    buf = (C.c_uint64 * (nb * nit * NPH))()
    nbo = C.c_int32(0)
    info = _abi.SolveInfo()
    E.solve_rtol(f, x, rtol=rtol)  # warm-up
    x.zero_()
    rc = L.pyomgpu_resident_trace(E._ctx, _ptr(f, E.shape), _ptr(x, E.shape, True), rtol, it0, nit, buf,
                                  C.byref(nbo), C.byref(info), _stream())
    _abi.check(rc)
    t = np.frombuffer(buf, dtype=np.uint64).reshape(nbo.value, nit, NPH).astype(np.int64)
    E.close()
    return t, info.as_dict(), lay


def summarise(t):
    ok = (t[:, :-1, :] > 0).all(axis=(0, 2))  # full iterations (the next one started too)
    t = t[:, :-1][:, ok[: t.shape[1] - 1]] if ok.any() else t
    out = {"blocks": int(t.shape[0]), "iterations": int(t.shape[1]), "intervals_ns": {}}
    for label, a, b in INTERVALS:
        d = (t[:, :, b] - t[:, :, a]).reshape(-1)
        out["intervals_ns"][label] = {"median": float(np.median(d)), "p90": float(np.percentile(d, 90)),
                                      "max": float(d.max())}
    period = np.diff(t[0, :, 0])
    out["iteration_ns"] = {"median": float(np.median(period)), "p90": float(np.percentile(period, 90))}
    # skew: spread over blocks of the moment each publishes its slot, and of the
    # moment each has acquired all slots
    for tag, ph in (("publish A", 11), ("acquire A", 12), ("publish B", 15), ("acquire B", 16)):
        s = t[:, :, ph] - t[:, :, ph].min(axis=0, keepdims=True)
        out[f"skew {tag} ns"] = {"median_of_max": float(np.median(s.max(axis=0))),
                                 "slowest_block_mode": int(np.bincount(s.argmax(axis=0)).argmax())}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--it0", type=int, default=400)
    ap.add_argument("--nit", type=int, default=64)
    ap.add_argument("--grid", default="c1", help="c1 (1440x720) or c3 (2048x1024)")
    ap.add_argument("--json", default=None)
    args = ap.parse_args()
    from pyom2_b200 import synth
    W = synth.config1() if args.grid == "c1" else synth.config3()
    t, info, lay = run(W, args.it0, args.nit)
    s = summarise(t)
    s["layout"] = {"npx": lay[0], "npy": lay[1], "points_per_thread": lay[2]}
    s["solve"] = {"iterations": info["iterations"], "device_ms": info["device_ms"]}
    print(json.dumps(s, indent=1))
    if args.json:
        with open(args.json, "w") as fh:
            json.dump(s, fh, indent=1)
        np.save(args.json.replace(".json", ".npy"), t)


if __name__ == "__main__":
    main()
