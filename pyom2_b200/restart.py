"""Restart interchange with pyOM2 for the external-mode state.

pyOM2 writes one unformatted sequential file per PE, ``restart_PE_00000.dta``
(for_src/main/restart.f90:1-93), and reads it back in ``read_restart``
(:95-190).  The external mode needs ``psi``, ``dpsi`` (all three levels: the
first guess uses them, :158-161) and ``dpsin`` from it, and its time step
reads ``u, v, du, dv, rho`` at ``tau``/``taum1``.  This module reads those
records from a file the Fortran model wrote, copies a file record by record
while replacing them (so a run can continue from the GPU solver's state), and
writes a file of the same structure with the records the external mode does
not own set to zero.

Record layout (one Fortran ``write`` statement = one record):

====  ==========================================================
 0    nx, ny, nz, itt                      (int32 x 4)
 1    is, ie, js, je = 1-onx, nx+onx, ...  (int32 x 4)
 2    rho(tau), rho(taum1)                 (each (nx+4, ny+4, nz) float64)
 3-6  Nsqr, Hd, int_drhodT, int_drhodS     (tau, taum1)
 7    dHd                                   (tau, taum1)
 8-11 temp, dtemp, salt, dsalt              (tau, taum1)
 12   u(tau), u(taum1)
 13   du(tau), du(taum1)
 14   v(tau), v(taum1)
 15   dv(tau), dv(taum1)
 16   w(tau), w(taum1)
 17   psi(taum1), psi(tau)                  (each (nx+4, ny+4))
 18   dpsi(taum1), dpsi(tau)                (enable_streamfunction only)
 19   dpsi(taup1)
 20   dpsin(1:nisle, tau), dpsin(1:nisle, taum1)
 ...  optional modules (eke, tke, idemix, ...), copied unchanged
====  ==========================================================

Sequential unformatted records are framed the gfortran way: a signed 4-byte
length before and after each record; a record longer than 2**31 - 9 bytes is
split into subrecords whose leading length is negative for every subrecord
but the last (and whose trailing length is negative for every subrecord but
the first).
"""
from __future__ import annotations

import struct

import numpy as np

_MAXSUB = 2**31 - 9  # largest subrecord payload gfortran writes


def read_records(path):
    """All records of a sequential unformatted file, as bytes."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos, n = 0, len(data)
    while pos < n:
        parts = []
        while True:
            if pos + 4 > n:
                raise ValueError(f"{path}: truncated record marker at byte {pos}")
            (lead,) = struct.unpack_from("<i", data, pos)
            size = abs(lead)
            end = pos + 4 + size
            if end + 4 > n:
                raise ValueError(f"{path}: truncated record at byte {pos}")
            parts.append(data[pos + 4:end])
            (trail,) = struct.unpack_from("<i", data, end)
            if abs(trail) != size:
                raise ValueError(f"{path}: record markers {lead} / {trail} disagree at byte {pos}")
            pos = end + 4
            if lead >= 0:
                break
        out.append(b"".join(parts))
    return out


def write_records(path, records, maxsub=_MAXSUB):
    with open(path, "wb") as f:
        for rec in records:
            chunks = [rec[i:i + maxsub] for i in range(0, len(rec), maxsub)] or [b""]
            for k, c in enumerate(chunks):
                lead = -len(c) if k < len(chunks) - 1 else len(c)
                trail = -len(c) if k > 0 else len(c)
                f.write(struct.pack("<i", lead))
                f.write(c)
                f.write(struct.pack("<i", trail))


def _arr(a):
    if type(a).__module__.startswith("torch"):
        a = a.detach().cpu().numpy()
    return np.asarray(a, dtype=np.float64)


def _f(a):
    return np.asfortranarray(_arr(a)).tobytes(order="F")


def _fields(rec, shape, count):
    n = int(np.prod(shape))
    v = np.frombuffer(rec, dtype="<f8")
    if v.size != n * count:
        raise ValueError(f"record holds {v.size} values, expected {count} x {shape}")
    return [np.reshape(v[k * n:(k + 1) * n], shape, order="F") for k in range(count)]


_IDX = {"rho": 2, "u": 12, "du": 13, "v": 14, "dv": 15, "w": 16}


def _check_header(recs, M):
    nx, ny, nz, itt = struct.unpack("<4i", recs[0])
    if (nx, ny, nz) != (M.nx, M.ny, M.nz):
        raise ValueError(f"restart dimensions {nx, ny, nz} do not match {M.nx, M.ny, M.nz}")
    bounds = struct.unpack("<4i", recs[1])
    want = (1 - M.onx, M.nx + M.onx, 1 - M.onx, M.ny + M.onx)
    if bounds != want:  # restart.f90:134-140
        raise ValueError(f"restart PE boundaries {bounds} do not match {want}")
    return itt


def read_external_state(path, M, enable_streamfunction=True, fields=("rho", "u", "du", "v", "dv")):
    """restart.f90:95-163 for the external mode: fills M.psi (taum1, tau),
    M.dpsi (all levels) and M.dpsin (tau, taum1), and the 3-D ``fields`` at
    tau and taum1.  Returns itt."""
    recs = read_records(path)
    itt = _check_header(recs, M)
    X, Y = M.shape2d
    s3 = (X, Y, M.nz)
    for name in fields:
        a, b = _fields(recs[_IDX[name]], s3, 2)
        arr = getattr(M, name)
        arr[..., M.tau - 1] = a
        arr[..., M.taum1 - 1] = b
    a, b = _fields(recs[17], (X, Y), 2)
    M.psi[..., M.taum1 - 1] = a
    M.psi[..., M.tau - 1] = b
    if enable_streamfunction:
        a, b = _fields(recs[18], (X, Y), 2)
        M.dpsi[..., M.taum1 - 1] = a
        M.dpsi[..., M.tau - 1] = b
        (c,) = _fields(recs[19], (X, Y), 1)
        M.dpsi[..., M.taup1 - 1] = c
        nisle = len(recs[20]) // 16
        if M.dpsin is None or M.dpsin.shape[0] != nisle:
            raise ValueError(f"restart holds {nisle} islands, the model {0 if M.dpsin is None else M.dpsin.shape[0]}")
        v = np.frombuffer(recs[20], dtype="<f8")
        M.dpsin[:, M.tau - 1] = v[:nisle]
        M.dpsin[:, M.taum1 - 1] = v[nisle:]
    return itt


def _external_records(M, enable_streamfunction, fields):
    t, tm = M.tau - 1, M.taum1 - 1
    out = {}
    for name in fields:
        a = _arr(getattr(M, name))
        out[_IDX[name]] = _f(a[..., t]) + _f(a[..., tm])
    psi = _arr(M.psi)
    out[17] = _f(psi[..., tm]) + _f(psi[..., t])
    if enable_streamfunction:
        dpsi = _arr(M.dpsi)
        out[18] = _f(dpsi[..., tm]) + _f(dpsi[..., t])
        out[19] = _f(dpsi[..., M.taup1 - 1])
        dpsin = _arr(M.dpsin) if M.dpsin is not None else np.zeros((0, 3))
        out[20] = dpsin[:, t].astype("<f8").tobytes() + dpsin[:, tm].astype("<f8").tobytes()
    return out


def update_restart(path_in, path_out, M, enable_streamfunction=True, fields=("u", "du", "v", "dv")):
    """Copy a pyOM2 restart file record by record, replacing psi, dpsi, dpsin
    and the 3-D ``fields`` with M's values (the state after GPU solves), so the
    Fortran model continues from it.  Every other record is copied unchanged."""
    recs = read_records(path_in)
    _check_header(recs, M)
    for k, rec in _external_records(M, enable_streamfunction, fields).items():
        if len(rec) != len(recs[k]):
            raise ValueError(f"record {k}: {len(rec)} bytes replace {len(recs[k])}")
        recs[k] = rec
    write_records(path_out, recs)


def write_restart(path, M, itt, enable_streamfunction=True, fields=("rho", "u", "du", "v", "dv", "w")):
    """A restart file with restart.f90:17-50's record structure (through
    dpsin) from M; records of fields the external mode does not hold
    (Nsqr, Hd, int_drhodT/S, dHd, temp, dtemp, salt, dsalt) are zero."""
    X, Y = M.shape2d
    n3 = X * Y * M.nz * 8
    recs = [struct.pack("<4i", M.nx, M.ny, M.nz, int(itt)),
            struct.pack("<4i", 1 - M.onx, M.nx + M.onx, 1 - M.onx, M.ny + M.onx)]
    recs += [bytes(2 * n3) for _ in range(2, 17)]
    have = [f for f in fields if getattr(M, f, None) is not None]
    for k, rec in _external_records(M, enable_streamfunction, have).items():
        if k < len(recs):
            recs[k] = rec
        else:
            recs.append(rec)
    write_records(path, recs)
