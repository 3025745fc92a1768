"""Seeded synthetic inputs for the external-mode solve.

pyOM2 builds the solver's inputs in ``calc_grid`` / ``calc_topo``
(for_src/main/numerics.f90:6-168,187-261) from user-set ``dxt/dyt/dzt`` and
``kbot``.  The functions ``u_centered_grid``, ``calc_grid`` and ``calc_topo``
below restate those routines (serial build, one PE) so that the metric arrays
``dxt,dxu,dyt,dyu,cost,cosu`` and the masks / depths ``hu,hv,hur,hvr`` have
exactly the layout and values the reference would hand to the solver.

No public data set is involved: every workload is generated from a seeded
``numpy.random.Generator(PCG64(seed))``.  Smooth fields are white noise
filtered with a Gaussian of the stated correlation length (in cells) and
rescaled to the stated rms.  The workloads:

* ``config0``   40x40, 2-degree sector 0-80E / 40S-40N, land ring + one 4x4
                island, 4000 m minus a 1500 m Gaussian ridge (8-cell width).
* ``config1``   1440x720, 0.25 x (160/720) degree, 80S-80N, cyclic in x,
                ~30 % land from thresholded smooth noise, 20 land masses,
                depth 500-5500 m.
* ``config3``   2048x1024 with the config1 recipe.
* ``config2``   64 closed basins, nx in [128,1024], ny in [128,768],
                10-40 % land, 0-12 interior islands each.
* ``config4``   256x256x20 re-entrant channel, 60S-30S, one 2000 m
                meridional ridge; a seeded sequence of momentum tendencies
                (pyom2_b200/sequence.py).

The right-hand side follows solve_streamfct.f90:39-53: a vertically
integrated forcing (fpx, fpy) is scaled by ``hur/hvr`` and its curl is the
streamfunction forcing ``forc``.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.ndimage as ndi

from .model import ModelState, DEGTOM, PI_F, ONX, RADIUS


# ----------------------------------------------------------------------------
# grid / topography set-up (numerics.f90)
# ----------------------------------------------------------------------------
def u_centered_grid(dyt):
    """numerics.f90:6-28.  Returns (dyu, yt, yu) for cell widths ``dyt``."""
    n = dyt.shape[0]
    yu = np.zeros(n)
    yt = np.zeros(n)
    dyu = np.zeros(n)
    for i in range(1, n):
        yu[i] = yu[i - 1] + dyt[i]
    yt[0] = yu[0] - dyt[0] * 0.5
    for i in range(1, n):
        yt[i] = 2 * yu[i - 1] - yt[i - 1]
    for i in range(0, n - 1):
        dyu[i] = yt[i + 1] - yt[i]
    dyu[n - 1] = 2 * dyt[n - 1] - dyu[max(0, n - 2)]
    return dyu, yt, yu


def _fill_1d_halo(a, n, cyclic):
    """Halo fill of a 1-D grid array as in numerics.f90:54-62 (Python index
    p = Fortran index f + 1, interior f = 1..n)."""
    for i in range(1, ONX + 1):
        if cyclic:
            a[n + i + 1] = a[i + 1]
            a[1 - i + 1] = a[n - i + 1 + 1]
        else:
            a[n + i + 1] = a[n + 1]
            a[1 - i + 1] = a[1 + 1]


def calc_grid(M: ModelState):
    """numerics.f90:34-168 restricted to what the external mode uses."""
    nx, ny = M.nx, M.ny
    P = lambda f: f + 1  # Fortran halo index -> Python index
    dxt = M.dxt.copy()
    dyt = M.dyt.copy()
    _fill_1d_halo(dxt, nx, M.enable_cyclic_x)
    _fill_1d_halo(dyt, ny, M.enable_cyclic_y)
    dxu, xt, xu = u_centered_grid(dxt)
    xt = xt - xu[P(1)] + M.x_origin
    xu = xu - xu[P(1)] + M.x_origin
    if M.enable_cyclic_x:
        for i in range(1, ONX + 1):
            xt[P(nx + i)] = xt[P(i)]
            xt[P(1 - i)] = xt[P(nx - i + 1)]
            xu[P(nx + i)] = xt[P(i)]          # numerics.f90:88 uses xt here
            xu[P(1 - i)] = xu[P(nx - i + 1)]
            dxu[P(nx + i)] = dxu[P(i)]
            dxu[P(1 - i)] = dxu[P(nx - i + 1)]
    dyu, yt, yu = u_centered_grid(dyt)
    yt = yt - yu[P(1)] + M.y_origin
    yu = yu - yu[P(1)] + M.y_origin
    if M.enable_cyclic_y:
        for j in range(1, ONX + 1):
            yt[P(ny + j)] = yt[P(j)]
            yt[P(1 - j)] = yt[P(ny - j + 1)]
            yu[P(ny + j)] = yt[P(j)]
            yu[P(1 - j)] = yu[P(ny - j + 1)]
            dyu[P(ny + j)] = dyu[P(j)]
            dyu[P(1 - j)] = dyu[P(ny - j + 1)]
    if M.coord_degree:
        dxt = dxt * DEGTOM
        dxu = dxu * DEGTOM
        dyt = dyt * DEGTOM
        dyu = dyu * DEGTOM
    M.xt[:], M.xu[:], M.dxt[:], M.dxu[:] = xt, xu, dxt, dxu
    M.yt[:], M.yu[:], M.dyt[:], M.dyu[:] = yt, yu, dyt, dyu
    dzw, zt, zw = u_centered_grid(M.dzt)
    M.dzw[:] = dzw
    M.zt[:] = zt - zw[-1]
    M.zw[:] = zw - zw[-1]
    if M.coord_degree:
        M.cost[:] = np.cos(yt / 180.0 * PI_F)
        M.cosu[:] = np.cos(yu / 180.0 * PI_F)
        # tan of the C library, element by element, as the Fortran intrinsic
        M.tantr[:] = [math.tan(y / 180.0 * PI_F) / RADIUS for y in yt]
    else:
        M.cost[:] = 1.0
        M.cosu[:] = 1.0
        M.tantr[:] = 0.0
    # box areas (numerics.f90:160-167)
    M.area_t[...] = (M.dxt[:, None] * M.cost[None, :]) * M.dyt[None, :]
    M.area_u[...] = (M.dxu[:, None] * M.cost[None, :]) * M.dyt[None, :]
    M.area_v[...] = (M.dxt[:, None] * M.cosu[None, :]) * M.dyu[None, :]
    M.area_z[...] = (M.dxu[:, None] * M.cosu[None, :]) * M.dyu[None, :]


def setcyclic_xy(M: ModelState, a):
    """parallel_none.f90:188-211 for a 2-D (or leading-2-D) array."""
    nx, ny = M.nx, M.ny
    if M.enable_cyclic_x:
        for i in range(1, ONX + 1):
            a[nx + i + 1] = a[i + 1]
            a[1 - i + 1] = a[nx - i + 1 + 1]
    if M.enable_cyclic_y:
        for j in range(1, ONX + 1):
            a[:, ny + j + 1] = a[:, j + 1]
            a[:, 1 - j + 1] = a[:, ny - j + 1 + 1]


def calc_topo(M: ModelState):
    """numerics.f90:187-261: close the domain, build masks T/U/V/Z/W and the
    column depths ``hu, hv`` with reciprocals ``hur, hvr``."""
    nx, ny, nz = M.nx, M.ny, M.nz
    kbot = M.kbot
    if not M.enable_cyclic_y:
        kbot[:, 0:2] = 0
        kbot[:, ny + 2:ny + 4] = 0
    if not M.enable_cyclic_x:
        kbot[0:2, :] = 0
        kbot[nx + 2:nx + 4, :] = 0
    setcyclic_xy(M, kbot)
    k = np.arange(1, nz + 1)[None, None, :]
    kb = kbot[:, :, None]
    maskT = np.where((kb != 0) & (kb <= k), 1.0, 0.0)
    setcyclic_xy(M, maskT)
    maskU = maskT.copy()
    maskU[:-1] = np.minimum(maskT[:-1], maskT[1:])
    setcyclic_xy(M, maskU)
    maskV = maskT.copy()
    maskV[:, :-1] = np.minimum(maskT[:, :-1], maskT[:, 1:])
    setcyclic_xy(M, maskV)
    maskZ = maskT.copy()
    maskZ[:-1, :-1] = np.minimum(np.minimum(maskT[:-1, :-1], maskT[:-1, 1:]), maskT[1:, :-1])
    setcyclic_xy(M, maskZ)
    M.maskT[...] = maskT
    M.maskU[...] = maskU
    M.maskV[...] = maskV
    M.maskZ[...] = maskZ
    maskW = maskT.copy()                          # numerics.f90:246-249
    maskW[:, :, :-1] = np.minimum(maskT[:, :, :-1], maskT[:, :, 1:])
    M.maskW[...] = maskW
    dzt = M.dzt[None, None, :]
    M.ht[...] = (maskT * dzt).sum(axis=2)
    M.hu[...] = 0.0
    M.hv[...] = 0.0
    for kk in range(nz):          # same summation order as numerics.f90:254-258
        M.hu += maskU[:, :, kk] * M.dzt[kk]
        M.hv += maskV[:, :, kk] * M.dzt[kk]
    M.hur[...] = 0.0
    M.hvr[...] = 0.0
    nzu = M.hu != 0.0
    nzv = M.hv != 0.0
    M.hur[nzu] = 1.0 / M.hu[nzu]
    M.hvr[nzv] = 1.0 / M.hv[nzv]


# ----------------------------------------------------------------------------
# random fields and land-mask post-processing
# ----------------------------------------------------------------------------
def smooth_field(rng, shape, sigma, cyclic=(False, False)):
    w = rng.standard_normal(shape)
    mode = tuple("wrap" if c else "reflect" for c in cyclic)
    return ndi.gaussian_filter(w, sigma, mode=mode)


_S8 = np.ones((3, 3), dtype=bool)
_S4 = ndi.generate_binary_structure(2, 1)


def _label_periodic(mask, structure, cyclic_x):
    """Connected components of ``mask`` (x = axis 0) with optional periodic x."""
    lab, n = ndi.label(mask, structure=structure)
    if not cyclic_x or n == 0:
        return lab, n
    parent = np.arange(n + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    nxl, nyl = mask.shape
    offs = (-1, 0, 1) if structure is _S8 else (0,)
    for dj in offs:
        j0, j1 = max(0, -dj), min(nyl, nyl - dj)
        a = lab[-1, j0:j1]
        b = lab[0, j0 + dj:j1 + dj]
        for p, q in zip(a[(a > 0) & (b > 0)], b[(a > 0) & (b > 0)]):
            rp, rq = find(p), find(q)
            if rp != rq:
                parent[max(rp, rq)] = min(rp, rq)
    roots = np.array([find(a) for a in range(n + 1)])
    uniq, inv = np.unique(roots, return_inverse=True)
    lab = inv[lab]
    return lab, len(uniq) - 1


def clean_land_mask(land, cyclic_x, keep_islands=None, rng=None, max_passes=50):
    """Make a T-cell land mask (interior nx x ny, x = axis 0) safe for pyOM2's
    island set-up (island_module.f90, streamfct_init.f90):

    * the domain is closed to the north/south by land rows (as calc_topo does);
    * enclosed lakes (ocean not 4-connected to the main ocean) are filled;
    * ocean cells 8-adjacent to two different land masses ("perimeter
      collisions", island_module.f90:219-249) are filled, merging the masses;
    * optionally only the ``keep_islands`` largest land masses that do not
      touch the outer boundary are kept (the rest become ocean).
    Returns the cleaned boolean land mask.
    """
    land = land.copy()
    nx, ny = land.shape
    for _ in range(max_passes):
        changed = False
        if cyclic_x:
            # pyOM2's isleperim treats columns 0..nx+1 as one periodic row of
            # nx+2 cells (island_module.f90:71-77,373-419), so land in column 1
            # or nx that does not cross the seam gets a second label that the
            # halo copy then erases (streamfct_init.f90:56-83 halts on it).
            # Keep the two seam columns identical so seam land always crosses.
            seam = land[0] | land[-1]
            if (seam != land[0]).any() or (seam != land[-1]).any():
                land[0] = seam
                land[-1] = seam
                changed = True
        ext = np.ones((nx, ny + 2), dtype=bool)           # closed N/S
        ext[:, 1:-1] = land
        if not cyclic_x:
            ext = np.pad(ext, ((1, 1), (0, 0)), constant_values=True)
        # lakes
        olab, no = _label_periodic(~ext, _S4, cyclic_x)
        if no > 1:
            sizes = np.bincount(olab.ravel())
            sizes[0] = 0
            keep = np.argmax(sizes)
            lake = (olab > 0) & (olab != keep)
            if lake.any():
                ext[lake] = True
                changed = True
        # collisions
        llab, nl = _label_periodic(ext, _S8, cyclic_x)
        pad_mode = "wrap" if cyclic_x else "edge"
        lp = np.pad(llab, ((1, 1), (0, 0)), mode=pad_mode)
        lp = np.pad(lp, ((0, 0), (1, 1)), mode="edge")
        nb = [lp[1 + di:1 + di + ext.shape[0], 1 + dj:1 + dj + ext.shape[1]]
              for di in (-1, 0, 1) for dj in (-1, 0, 1) if (di, dj) != (0, 0)]
        nb = np.stack(nb, axis=0).astype(np.int64)
        big = np.where(nb > 0, nb, np.iinfo(np.int64).max)
        mn = big.min(axis=0)
        mx = np.where(nb > 0, nb, -1).max(axis=0)
        coll = (~ext) & (mx > 0) & (mn != mx)
        if coll.any():
            ext[coll] = True
            changed = True
        if cyclic_x:
            land = ext[:, 1:-1]
        else:
            land = ext[1:-1, 1:-1]
        if not changed:
            break
    else:
        raise RuntimeError("land mask clean-up did not converge")
    if keep_islands is not None:
        ext = np.ones((nx, ny + 2), dtype=bool)
        ext[:, 1:-1] = land
        if not cyclic_x:
            ext = np.pad(ext, ((1, 1), (0, 0)), constant_values=True)
        llab, nl = _label_periodic(ext, _S8, cyclic_x)
        boundary_labels = set(np.unique(llab[:, 0])) | set(np.unique(llab[:, -1]))
        if not cyclic_x:
            boundary_labels |= set(np.unique(llab[0, :])) | set(np.unique(llab[-1, :]))
        boundary_labels.discard(0)
        sizes = np.bincount(llab.ravel(), minlength=nl + 1)
        inner = [l for l in range(1, nl + 1) if l not in boundary_labels]
        inner.sort(key=lambda l: -sizes[l])
        drop = inner[keep_islands:]
        if drop:
            ext[np.isin(llab, drop)] = False
        land = ext[:, 1:-1] if cyclic_x else ext[1:-1, 1:-1]
    return land


# ----------------------------------------------------------------------------
# right-hand side (solve_streamfct.f90:39-53)
# ----------------------------------------------------------------------------
def forcing_from_fp(M: ModelState, fpx, fpy):
    """``forc`` = curl of (fpx, fpy) on the interior, solve_streamfct.f90:49-53."""
    nx, ny = M.nx, M.ny
    forc = np.zeros(M.shape2d, order="F")
    I = slice(2, nx + 2)
    J = slice(2, ny + 2)
    cosu = M.cosu[J][None, :]
    dxu = M.dxu[I][:, None]
    dyu = M.dyu[J][None, :]
    cost_j = M.cost[J][None, :]
    cost_jp = M.cost[3:ny + 3][None, :]
    forc[I, J] = ((fpy[3:nx + 3, J] - fpy[I, J]) / (cosu * dxu)
                  - (cost_jp * fpx[I, 3:ny + 3] - cost_j * fpx[I, J]) / (cosu * dyu))
    return forc


def random_fp(M: ModelState, rng, sigma=5.0, rms=1e-7):
    """Vertically integrated forcing (fpx, fpy) already multiplied by hur/hvr
    as in solve_streamfct.f90:39-48."""
    cyc = (M.enable_cyclic_x, M.enable_cyclic_y)
    gx = smooth_field(rng, M.shape2d, sigma, cyc)
    gy = smooth_field(rng, M.shape2d, sigma, cyc)
    mu = M.maskU[:, :, -1]
    mv = M.maskV[:, :, -1]
    for g, m in ((gx, mu), (gy, mv)):
        ocean = m > 0
        s = np.sqrt(np.mean(g[ocean] ** 2)) if ocean.any() else 1.0
        g *= rms / s
    fpx = np.asfortranarray(gx * mu * M.hur)
    fpy = np.asfortranarray(gy * mv * M.hvr)
    setcyclic_xy(M, fpx)
    setcyclic_xy(M, fpy)
    return fpx, fpy


def _kbot_from_depth(H, dz, nz):
    n = np.clip(np.rint(H / dz).astype(np.int64), 1, nz)
    return (nz - n + 1).astype(np.int32)


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
class Workload:
    """A model state with its solver forcing (``forc``, ``fpx``, ``fpy``)."""

    def __init__(self, name, M, fpx, fpy, forc, seed, meta=None):
        self.name, self.M, self.fpx, self.fpy, self.forc = name, M, fpx, fpy, forc
        self.seed = seed
        self.meta = meta or {}


def config0(seed: int = 1000) -> Workload:
    """40x40 2-degree sector, land ring + one 4x4 island (nisle = 2)."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    nx = ny = 40
    nz = 20
    M = ModelState(nx, ny, nz, enable_cyclic_x=False, coord_degree=True)
    M.dxt[2:nx + 2] = 2.0
    M.dyt[2:ny + 2] = 2.0
    M.x_origin, M.y_origin = 0.0, -40.0
    M.dzt[:] = 4000.0 / nz
    calc_grid(M)
    i = np.arange(1, nx + 1, dtype=np.float64)
    ic = 0.5 * (nx + 1) + rng.uniform(-2.0, 2.0)
    H = 4000.0 - 1500.0 * np.exp(-((i - ic) ** 2) / (2.0 * 8.0 ** 2))
    kb = _kbot_from_depth(H, M.dzt[0], nz)
    M.kbot[2:nx + 2, 2:ny + 2] = kb[:, None]
    # land ring on the outermost interior rows/columns, Fortran 1 and nx/ny
    M.kbot[2, :] = 0
    M.kbot[nx + 1, :] = 0
    M.kbot[:, 2] = 0
    M.kbot[:, ny + 1] = 0
    c = nx // 2  # centred 4x4 block, Fortran i,j = 19..22
    M.kbot[c + 1 - 1:c + 1 + 3, c + 1 - 1:c + 1 + 3] = 0
    calc_topo(M)
    fpx, fpy = random_fp(M, rng, sigma=5.0, rms=1e-7)
    forc = forcing_from_fp(M, fpx, fpy)
    return Workload("c0_40x40", M, fpx, fpy, forc, seed)


def _global_like(nx, ny, lat0, lat1, seed, n_land_masses, land_frac=0.30,
                 mask_sigma=None, depth_sigma=None, nz=20, rhs_sigma=5.0,
                 name="global"):
    rng = np.random.default_rng(np.random.PCG64(seed))
    M = ModelState(nx, ny, nz, enable_cyclic_x=True, coord_degree=True)
    M.dxt[2:nx + 2] = 360.0 / nx
    M.dyt[2:ny + 2] = (lat1 - lat0) / ny
    M.x_origin, M.y_origin = 0.0, float(lat0)
    M.dzt[:] = 5500.0 / nz
    calc_grid(M)
    ms = mask_sigma if mask_sigma is not None else nx / 72.0
    noise = smooth_field(rng, (nx, ny), ms, (True, False))
    land = noise < np.quantile(noise, land_frac)
    # interior land masses = all masses minus the northern and southern coasts
    land = clean_land_mask(land, cyclic_x=True, keep_islands=max(0, n_land_masses - 2))
    ds = depth_sigma if depth_sigma is not None else nx / 60.0
    d = smooth_field(rng, (nx, ny), ds, (True, False))
    d = (d - d.min()) / (d.max() - d.min())
    H = 500.0 + 5000.0 * d
    kb = _kbot_from_depth(H, M.dzt[0], nz)
    kb[land] = 0
    M.kbot[2:nx + 2, 2:ny + 2] = kb
    calc_topo(M)
    fpx, fpy = random_fp(M, rng, sigma=rhs_sigma, rms=1e-7)
    forc = forcing_from_fp(M, fpx, fpy)
    return Workload(name, M, fpx, fpy, forc, seed,
                    meta={"land_fraction": float(land.mean())})


def config1(seed: int = 1001, nx=1440, ny=720) -> Workload:
    """1440x720, 80S-80N, cyclic x, ~30 % land, 20 land masses."""
    return _global_like(nx, ny, -80.0, 80.0, seed, n_land_masses=20,
                        name=f"c1_{nx}x{ny}")


def config3(seed: int = 1003, nx=2048, ny=1024) -> Workload:
    """2048x1024 with the config1 recipe."""
    return _global_like(nx, ny, -80.0, 80.0, seed, n_land_masses=20,
                        name=f"c3_{nx}x{ny}")


def config4(seed: int = 1004, nx=256, ny=256, nz=20, lon_extent=64.0) -> Workload:
    """Re-entrant channel: cyclic in x, 64 degrees long (0.25 degree cells at
    nx = 256), 60S-30S, closed to
    the north and south (calc_topo's land rows, so the walls are the two land
    masses and the channel transport is the one island unknown), 4000 m deep
    with one meridional ridge 2000 m high (Gaussian, 8-cell half width) at a
    seeded longitude.  The time-dependent inputs come from
    :class:`pyom2_b200.sequence.TendencySequence`."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    M = ModelState(nx, ny, nz, enable_cyclic_x=True, coord_degree=True)
    M.dxt[2:nx + 2] = lon_extent / nx  # 0.25 degree at the default size
    M.dyt[2:ny + 2] = 30.0 / ny
    M.x_origin, M.y_origin = 0.0, -60.0
    M.dzt[:] = 4000.0 / nz
    M.dt_mom = 1800.0
    M.congr_max_iterations = 20000  # the reference's channel set-ups raise it too (py_config/acc2.py:30)
    calc_grid(M)
    i = np.arange(1, nx + 1, dtype=np.float64)
    ic = nx * rng.uniform(0.3, 0.7)
    H = 4000.0 - 2000.0 * np.exp(-((i - ic) / 8.0) ** 2)
    M.kbot[2:nx + 2, 2:ny + 2] = _kbot_from_depth(H, M.dzt[0], nz)[:, None]
    calc_topo(M)
    forc = np.zeros(M.shape2d, order="F")
    return Workload(f"c4_{nx}x{ny}x{nz}", M, None, None, forc, seed, meta={"ridge_i": float(ic)})


def basin(nx, ny, seed, land_frac, n_islands, nz=20, lat0=-60.0) -> Workload:
    """Closed basin (no cyclic wrap) used for the batched set."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    M = ModelState(nx, ny, nz, enable_cyclic_x=False, coord_degree=True)
    dlon = 0.25
    dlat = min(0.25, 100.0 / ny)
    M.dxt[2:nx + 2] = dlon
    M.dyt[2:ny + 2] = dlat
    M.x_origin, M.y_origin = 0.0, float(lat0)
    M.dzt[:] = 5500.0 / nz
    calc_grid(M)
    noise = smooth_field(rng, (nx, ny), max(4.0, max(nx, ny) / 40.0), (False, False))
    land = noise < np.quantile(noise, land_frac)
    land = clean_land_mask(land, cyclic_x=False, keep_islands=n_islands)
    d = smooth_field(rng, (nx, ny), max(nx, ny) / 50.0, (False, False))
    d = (d - d.min()) / (d.max() - d.min())
    kb = _kbot_from_depth(500.0 + 5000.0 * d, M.dzt[0], nz)
    kb[land] = 0
    M.kbot[2:nx + 2, 2:ny + 2] = kb
    calc_topo(M)
    fpx, fpy = random_fp(M, rng, sigma=5.0, rms=1e-7)
    forc = forcing_from_fp(M, fpx, fpy)
    return Workload(f"basin_{nx}x{ny}", M, fpx, fpy, forc, seed,
                    meta={"land_fraction": float(land.mean())})


def config2(seed: int = 1002, count: int = 64, scale: float = 1.0):
    """64 independent basins with sizes from U[128..1024] x U[128..768].
    ``scale`` < 1 shrinks every grid (used for CPU-sized tests)."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    out = []
    for m in range(count):
        nx = int(rng.integers(128, 1025) * scale)
        ny = int(rng.integers(128, 769) * scale)
        nx, ny = max(nx, 16), max(ny, 16)
        lf = float(rng.uniform(0.10, 0.40))
        ni = int(rng.integers(0, 13))
        out.append(basin(nx, ny, seed * 1000 + m, lf, ni))
    return out


# ----------------------------------------------------------------------------
# non-hydrostatic pressure (non_hydrostatic.f90)
# ----------------------------------------------------------------------------
def nonhydro_forcing(M: ModelState, u, v, w, dt_mom):
    """Forcing of the non-hydrostatic pressure solve from the provisional
    velocities (u, v, w) at taup1, non_hydrostatic.f90:26-36: horizontal
    divergence on the interior, plus the vertical difference of w, over dt_mom."""
    nx, ny, nz = M.nx, M.ny, M.nz
    forc = np.zeros(M.shape2d + (nz,), order="F")
    I = slice(2, nx + 2)
    J = slice(2, ny + 2)
    cost = M.cost[J][None, :, None]
    cosu = M.cosu[J][None, :, None]
    cosum = M.cosu[1:ny + 1][None, :, None]
    dxt = M.dxt[I][:, None, None]
    dyt = M.dyt[J][None, :, None]
    forc[I, J] = ((u[I, J] - u[1:nx + 1, J]) / (cost * dxt)
                  + (cosu * v[I, J] - cosum * v[I, 1:ny + 1]) / (cost * dyt))
    forc[:, :, 0] = forc[:, :, 0] + w[:, :, 0] / M.dzt[0]
    for k in range(1, nz):
        forc[:, :, k] = forc[:, :, k] + (w[:, :, k] - w[:, :, k - 1]) / M.dzt[k]
    return np.asfortranarray(forc / dt_mom)


class Workload3D:
    """A model state with the forcing and first guess of one non-hydrostatic
    pressure solve."""

    def __init__(self, name, M, forc, p0, seed, meta=None):
        self.name, self.M, self.forc, self.p0, self.seed = name, M, forc, p0, seed
        self.meta = meta or {}


def nonhydro_tank(nx, ny, nz, seed, cyclic_x=False, dx=0.01, slope=True, vel_rms=1e-3, first_guess=False):
    """Cartesian tank (dx = dy = dz), closed walls (or re-entrant in x), a
    shelf over the first quarter in x falling linearly to the full depth, with
    seeded smooth roughness on the slope.  The forcing is the divergence of a
    seeded smooth masked velocity field (rigid lid, w(nz) = 0), so it lies in
    the range of the operator.  ``first_guess`` adds a smooth nonzero start
    (the reference starts from 2 p(tau) - p(taum1))."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    M = ModelState(nx, ny, nz, enable_cyclic_x=cyclic_x, coord_degree=False)
    M.dxt[2:nx + 2] = dx
    M.dyt[2:ny + 2] = dx
    M.dzt[:] = dx
    M.dt_mom = 0.25 * dx / 0.01
    calc_grid(M)
    H0 = dx * nz
    if slope and nz > 2:
        i = np.arange(1, nx + 1, dtype=np.float64)
        shelf = 0.25 * H0
        edge = max(1, nx // 4)
        H = np.where(i <= edge, shelf, shelf + (H0 - shelf) * (i - edge) / max(1, nx - edge))
        rough = smooth_field(rng, (nx, ny), max(2.0, nx / 16.0), (cyclic_x, False))
        rough = rough / (np.abs(rough).max() + 1e-300)
        Hij = np.clip(H[:, None] + 0.1 * H0 * rough * (i[:, None] > edge), dx, H0)
        kb = _kbot_from_depth(Hij, dx, nz)
    else:
        kb = np.ones((nx, ny), dtype=np.int32)
    M.kbot[2:nx + 2, 2:ny + 2] = kb
    calc_topo(M)
    shape3 = M.shape2d + (nz,)
    cyc = (cyclic_x, False, False)
    sig = (max(1.0, nx / 16.0), max(1.0, ny / 16.0), max(1.0, nz / 8.0))
    vel = []
    for m in (M.maskU, M.maskV, M.maskW):
        f = smooth_field(rng, shape3, sig, cyc)
        f *= vel_rms / (np.sqrt(np.mean(f ** 2)) + 1e-300)
        vel.append(np.asfortranarray(f * m))
    u, v, w = vel
    w[:, :, nz - 1] = 0.0
    for a in (u, v, w):
        setcyclic_xy(M, a)
    forc = nonhydro_forcing(M, u, v, w, M.dt_mom)
    p0 = np.zeros(shape3, order="F")
    if first_guess:
        g = smooth_field(rng, shape3, sig, cyc)
        p0 = np.asfortranarray(g * M.maskT * 1e-3)
        setcyclic_xy(M, p0)
    return Workload3D(f"tank_{nx}x{ny}x{nz}", M, forc, p0, seed)


def nonhydro_state(W: Workload3D, seed: int, vel_rms=1e-3):
    """Fill the model arrays that solve_non_hydrostatic reads (u, v, w at
    the three time levels, dw at tau and taum1, dw_mix, p_non_hydro at tau and
    taum1) with seeded smooth masked fields; w is zero at the rigid lid (k =
    nz), so the forcing the step builds is consistent."""
    M = W.M
    rng = np.random.default_rng(np.random.PCG64(seed))
    shape3 = M.shape2d + (M.nz,)
    cyc = (M.enable_cyclic_x, M.enable_cyclic_y, False)
    sig = (max(1.0, M.nx / 16.0), max(1.0, M.ny / 16.0), max(1.0, M.nz / 8.0))

    def field(mask, rms):
        f = smooth_field(rng, shape3, sig, cyc)
        f *= rms / (np.sqrt(np.mean(f ** 2)) + 1e-300)
        f = np.asfortranarray(f * mask)
        setcyclic_xy(M, f)
        return f

    for lev in range(3):
        M.u[..., lev] = field(M.maskU, vel_rms)
        M.v[..., lev] = field(M.maskV, vel_rms)
        M.w[..., lev] = field(M.maskW, vel_rms)
        M.dw[..., lev] = field(M.maskW, vel_rms * 1e-3)
        M.p_non_hydro[..., lev] = field(M.maskT, 1e-4)
    M.w[:, :, M.nz - 1, :] = 0.0
    M.dw_mix[...] = field(M.maskW, vel_rms * 1e-4)
    return W


WORKLOADS = {"c0": config0, "c1": config1, "c3": config3}
