"""Restart interchange (restart.f90:1-190): gfortran sequential unformatted
framing, the record layout the external mode reads and writes, and copying a
foreign restart file while replacing only the external-mode records."""
import struct

import numpy as np
import pytest

from pyom2_b200 import restart, synth
from pyom2_b200.model import ModelState


def small_model(nisle=3):
    W = synth.config0()
    M = W.M
    M.allocate_islands(nisle, 4)
    rng = np.random.default_rng(0)
    for n in ("rho", "u", "du", "v", "dv", "w", "psi", "dpsi", "dpsin"):
        a = getattr(M, n)
        a[...] = rng.standard_normal(a.shape)
    return M


def test_record_framing_and_subrecords(tmp_path):
    recs = [b"", b"abc", bytes(range(256)) * 3]
    p = tmp_path / "f.dta"
    restart.write_records(p, recs, maxsub=100)   # forces subrecords
    raw = p.read_bytes()
    # first record: empty payload between two zero markers
    assert raw[:8] == struct.pack("<ii", 0, 0)
    # second: 3-byte record
    assert raw[8:19] == struct.pack("<i", 3) + b"abc" + struct.pack("<i", 3)
    # third: 768 bytes in 8 subrecords: leading markers negative except the last, trailing except the first
    (lead,) = struct.unpack_from("<i", raw, 19)
    assert lead == -100
    assert restart.read_records(p) == recs
    restart.write_records(p, recs)
    assert restart.read_records(p) == recs


def test_header_bytes(tmp_path):
    M = small_model()
    p = tmp_path / "restart_PE_00000.dta"
    restart.write_restart(p, M, itt=17)
    raw = p.read_bytes()
    assert raw[:24] == struct.pack("<i4ii", 16, M.nx, M.ny, M.nz, 17, 16)
    assert raw[24:48] == struct.pack("<i4ii", 16, -1, M.nx + 2, -1, M.ny + 2, 16)
    recs = restart.read_records(p)
    X, Y = M.shape2d
    assert len(recs) == 21
    assert len(recs[2]) == 2 * X * Y * M.nz * 8 and len(recs[17]) == 2 * X * Y * 8
    assert len(recs[20]) == 2 * M.nisle * 8


def test_write_then_read_round_trip(tmp_path):
    M = small_model()
    p = tmp_path / "r.dta"
    restart.write_restart(p, M, itt=5)
    M2 = ModelState(M.nx, M.ny, M.nz)
    M2.allocate_islands(M.nisle, 4)
    M2.taum1, M2.tau, M2.taup1 = M.taum1, M.tau, M.taup1
    assert restart.read_external_state(p, M2) == 5
    assert np.array_equal(M2.dpsi, M.dpsi)  # all three levels: the first guess needs them (restart.f90:160)
    for n in ("psi", "dpsin"):               # tau and taum1 only
        for t in (M.tau, M.taum1):
            assert np.array_equal(getattr(M2, n)[..., t - 1], getattr(M, n)[..., t - 1]), n
    for n in ("rho", "u", "du", "v", "dv"):
        for t in (M.tau, M.taum1):
            assert np.array_equal(getattr(M2, n)[..., t - 1], getattr(M, n)[..., t - 1]), n


def test_update_keeps_foreign_records(tmp_path):
    M = small_model()
    X, Y = M.shape2d
    rng = np.random.default_rng(1)
    n3, n2 = X * Y * M.nz * 8, X * Y * 8
    foreign = [struct.pack("<4i", M.nx, M.ny, M.nz, 99), struct.pack("<4i", -1, M.nx + 2, -1, M.ny + 2)]
    foreign += [rng.bytes(2 * n3) for _ in range(2, 17)]
    foreign += [rng.bytes(2 * n2), rng.bytes(2 * n2), rng.bytes(n2), rng.bytes(2 * M.nisle * 8)]
    foreign += [rng.bytes(2 * n3), rng.bytes(123)]  # optional modules (eke, ...)
    src, dst = tmp_path / "in.dta", tmp_path / "out.dta"
    restart.write_records(src, foreign)
    restart.update_restart(src, dst, M)
    out = restart.read_records(dst)
    replaced = {12, 13, 14, 15, 17, 18, 19, 20}
    for k, (a, b) in enumerate(zip(foreign, out)):
        assert (a != b) == (k in replaced), k
    M2 = ModelState(M.nx, M.ny, M.nz)
    M2.allocate_islands(M.nisle, 4)
    assert restart.read_external_state(dst, M2, fields=("u", "du", "v", "dv")) == 99
    assert np.array_equal(M2.dpsi, M.dpsi) and np.array_equal(M2.dpsin[:, [M.tau - 1, M.taum1 - 1]],
                                                               M.dpsin[:, [M.tau - 1, M.taum1 - 1]])


def test_mismatch_is_an_error(tmp_path):
    M = small_model()
    p = tmp_path / "r.dta"
    restart.write_restart(p, M, itt=1)
    M2 = ModelState(M.nx + 1, M.ny, M.nz)
    with pytest.raises(ValueError):
        restart.read_external_state(p, M2)
    M3 = ModelState(M.nx, M.ny, M.nz)
    M3.allocate_islands(M.nisle + 1, 4)
    with pytest.raises(ValueError):
        restart.read_external_state(p, M3)
