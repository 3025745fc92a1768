"""The on-chip-resident streamfunction CG kernels (csrc/cg_res.cu: two
reductions per iteration, and one with A p by recurrence and (p, Ap) by its
exact expansion) against the
CPU oracle and against the tiled kernel (csrc/cg_ref.cu) on the same inputs.

Tolerances: both kernels run congrad_streamfunction's algorithm in FP64 with
tree-ordered dot products (different orders), so converged solutions agree
with the oracle and with each other to 1e-10 relative and iteration counts
within one; the reference's status paths (max_it, NaN, time-out) are exact.
"""
import numpy as np
import pytest

from pyom2_b200 import _abi, synth
from pyom2_b200.external import ExternalMode

pytestmark = pytest.mark.gpu

RTOL_SOL = 1e-10


def it_tol(kernel, it_ref):
    """Iteration-count tolerance: the kernels with the reference's recurrences
    stop within one iteration of the oracle; the single-reduction form computes
    A p by recurrence and (p, Ap) by expansion, so its iterates drift at rounding level and the
    reference's extrapolated stopping estimate may cross its threshold a few
    iterations apart (the converged solution is held to RTOL_SOL all the same)."""
    return max(3, it_ref // 100) if kernel == "resident1" else 1


def rel(a, b, mask=None):
    a, b = np.asarray(a), np.asarray(b)
    if mask is not None:
        a, b = a[mask], b[mask]
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / n if n > 0 else np.linalg.norm(a - b)


WORLDS = {
    "c0": lambda: synth.config0(),
    "cyclic96": lambda: synth._global_like(96, 48, -80.0, 80.0, 13, n_land_masses=6, mask_sigma=4.0,
                                           depth_sigma=4.0, name="small"),
    "cyclic200": lambda: synth._global_like(200, 100, -80.0, 80.0, 9, n_land_masses=10, mask_sigma=4.0,
                                            depth_sigma=4.0, name="small"),
    "basin130": lambda: synth.basin(130, 70, 302, 0.25, 6),
    "channel96": lambda: synth.config4(1004, nx=96, ny=96, nz=4),
}


def setup(name, oracle_lib, kernel):
    W = WORLDS[name]()
    O = oracle_lib.Oracle(W.M.copy())
    O.streamfunction_init(maxipp=10**6, maxq=10**6)
    E = ExternalMode(W.M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6)
    E.set_cg_kernel(kernel)
    return W, O, E


@pytest.mark.parametrize("kernel", ["resident1", "resident", "tiled"])
@pytest.mark.parametrize("name", list(WORLDS))
def test_congrad_streamfunction_matches_oracle(oracle_lib, name, kernel):
    W, O, E = setup(name, oracle_lib, kernel)
    cf = O.make_coeff_streamfunction()
    rng = np.random.default_rng(11)
    sol0 = np.asfortranarray(rng.standard_normal(W.M.shape2d) * 1e3)
    so = sol0.copy(order="F")
    ro = O.congrad_streamfunction(cf, W.forc, so)
    sg = sol0.copy(order="F")
    it, conv, info = E.congrad_streamfunction(W.forc, sg)
    print(f"{name} {kernel}: iterations {it} (oracle {ro['iterations']}), rel {rel(sg, so):.2e}")
    assert rel(sg, so) < RTOL_SOL
    assert conv == ro["converged"] and abs(it - ro["iterations"]) <= it_tol(kernel, ro["iterations"]), (
        it, ro["iterations"])
    # halo as the reference leaves it (set once at entry)
    assert rel(sg[:2], so[:2]) < RTOL_SOL or np.array_equal(sg[:2], so[:2])


@pytest.mark.parametrize("name", ["c0", "cyclic200"])
def test_solve_rtol_resident(oracle_lib, name):
    W, O, E = setup(name, oracle_lib, "resident")
    sol = np.zeros(W.M.shape2d, order="F")
    info = E.solve_rtol(W.forc, sol, rtol=1e-10, precision=_abi.PREC_F64)
    assert info["status"] == 0 and info["rel_residual"] <= 1e-10, info
    cf = O.make_coeff_streamfunction()
    Z = O.make_inv_sfc(cf)
    assert O.rel_residual(cf, Z, W.forc, sol) <= 1.5e-10


@pytest.mark.parametrize("name", ["c0", "cyclic200", "basin130", "channel96"])
def test_mixed_precision_on_the_fp32_resident_kernel(oracle_lib, name):
    """solve_rtol with FP32 correction solves, which run on the FP32 resident
    kernel where the grid fits (FP32 fields, FP64 partial sums): the FP64
    true residual reaches rtol, the oracle's residual of the solution agrees,
    and the solution equals the one of the pipelined tile kernel's
    corrections (set_cg_kernel "tiled") to 1e-9 relative."""
    W, O, E = setup(name, oracle_lib, "auto")
    assert E.resident_layout(fp32=True) is not None
    sol = np.zeros(W.M.shape2d, order="F")
    info = E.solve_rtol(W.forc, sol, rtol=1e-10, precision=_abi.PREC_F32)
    assert info["status"] == 0 and info["rel_residual"] <= 1e-10, info
    cf = O.make_coeff_streamfunction()
    assert O.rel_residual(cf, O.make_inv_sfc(cf), W.forc, sol) <= 1.5e-10
    E.set_cg_kernel("tiled")
    s2 = np.zeros(W.M.shape2d, order="F")
    i2 = E.solve_rtol(W.forc, s2, rtol=1e-10, precision=_abi.PREC_F32)
    E.set_cg_kernel("auto")
    assert i2["status"] == 0
    assert rel(sol, s2) < 1e-9


def test_fp32_resident_fits_twice_the_grid():
    """2048 x 1024 does not fit the FP64 resident kernel but fits the FP32
    one at 32 points per thread; its mixed-precision solve reaches the FP64
    residual and agrees with the FP64 tiled solve."""
    W = synth.config3()
    E = ExternalMode(W.M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6, psin_rtol=1e-12, psin_weighted=True)
    assert E.resident_layout() is None
    npx, npy, p = E.resident_layout(fp32=True)
    assert p == 32 and npx * npy <= 148
    sol = np.zeros(W.M.shape2d, order="F")
    info = E.solve_rtol(W.forc, sol, rtol=1e-10, precision=_abi.PREC_F32)
    assert info["status"] == 0 and info["rel_residual"] <= 1e-10, info
    s64 = np.zeros(W.M.shape2d, order="F")
    i64 = E.solve_rtol(W.forc, s64, rtol=1e-10, precision=_abi.PREC_F64)
    assert i64["status"] == 0
    assert rel(sol, s64) < 1e-8


def test_headline_grid_layout_and_kernels_agree():
    """1440 x 720 (20 islands): 9 x 16 pieces of at most 160 x 45 points, 16
    points per thread (the cut with the least estimated iteration time); the
    resident kernels (two reductions and one per
    iteration) and the tiled kernel reach the same solution and the same
    iteration count within one."""
    W = synth.config1()
    E = ExternalMode(W.M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6)
    assert E.resident_layout() == (9, 16, 16)
    out = {}
    for kernel in ("tiled", "resident", "resident1"):
        E.set_cg_kernel(kernel)
        sol = np.zeros(W.M.shape2d, order="F")
        info = E.solve_rtol(W.forc, sol, rtol=1e-10, precision=_abi.PREC_F64)
        assert info["status"] == 0 and info["rel_residual"] <= 1e-10, (kernel, info)
        out[kernel] = (sol, info)
    st, it_t = out["tiled"]
    for kernel in ("resident", "resident1"):
        sr, it_r = out[kernel]
        assert abs(it_t["iterations"] - it_r["iterations"]) <= it_tol(kernel, it_t["iterations"]), kernel
        assert rel(sr, st) < 1e-8, kernel
    print("1440x720 device ms: " + ", ".join(f"{k} {out[k][1]['device_ms']:.2f}" for k in out))


@pytest.mark.parametrize("kernel", ["resident1", "resident"])
def test_reruns_are_bit_identical(kernel):
    W = WORLDS["cyclic200"]()
    E = ExternalMode(W.M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6)
    E.set_cg_kernel(kernel)
    a = np.zeros(W.M.shape2d, order="F")
    b = np.zeros(W.M.shape2d, order="F")
    ia = E.congrad_streamfunction(W.forc, a)[0]
    ib = E.congrad_streamfunction(W.forc, b)[0]
    assert ia == ib and np.array_equal(a, b)


@pytest.mark.parametrize("kernel", ["resident1", "resident", "tiled"])
def test_status_paths(oracle_lib, kernel):
    W, O, E = setup("c0", oracle_lib, kernel)
    bad = W.forc.copy(order="F")
    bad[10, 10] = np.nan
    with pytest.raises(_abi.PyOMGPUError) as e:
        E.congrad_streamfunction(bad, np.zeros(W.M.shape2d, order="F"))
    assert e.value.code == _abi.NAN
    with pytest.warns(RuntimeWarning):
        it, conv, info = E.congrad_streamfunction(W.forc, np.zeros(W.M.shape2d, order="F"), max_it=3)
    assert it == 4 and not conv and info["status"] == _abi.MAXITER
    E.set_sync_timeout(1e-3)
    E.inject_barrier_stall(True)
    with pytest.raises(_abi.PyOMGPUError) as e:
        E.congrad_streamfunction(W.forc, np.zeros(W.M.shape2d, order="F"))
    assert e.value.code == _abi.TIMEOUT
    E.set_sync_timeout(2.0)
    s = np.zeros(W.M.shape2d, order="F")
    it, conv, _ = E.congrad_streamfunction(W.forc, s)  # the context is still usable
    assert conv and it > 10


def test_too_large_grid_is_refused():
    W = synth.config3()  # 2048 x 1024: pieces do not fit on chip
    E = ExternalMode(W.M)
    assert E.resident_layout() is None
    with pytest.raises(_abi.PyOMGPUError) as e:
        E.set_cg_kernel("resident")
    assert e.value.code == _abi.EINVAL
    E.set_cg_kernel("auto")
