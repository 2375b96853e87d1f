"""Seeded synthetic SFINCS workloads written as the reference's own input files.

No public benchmark exists for the time-stepping core, so the named workloads
are generated here: a ``sfincs.inp`` plus the binary index/mask/depth files
(``sfincs_domain.f90:250-321,1672-1676`` stream-binary layout), ASCII boundary
(``bnd``/``bzs``, ``sfincs_boundaries.f90:62-98``), rain (``prcfile``,
``sfincs_meteo.f90`` read at ``:116-131`` of the meteo reader) and wind
(``wndfile``) time series, and a netCDF-3 subgrid table file whose variables
are the ones ``sfincs_subgrid.F90:102-122`` reads.

Array conventions: a regular grid is an ``(nmax, mmax)`` numpy array indexed
``[n-1, m-1]`` with ``n`` along y (rows, south to north) and ``m`` along x.  The
reference compacts active cells with ``n`` fastest, ``index=(m-1)*nmax+n``
(``sfincs_domain.f90:235-240``), i.e. Fortran order of the ``(nmax, mmax)`` array.

The subgrid tables are built by this project's own builder (the upstream
HydroMT-SFINCS builder is not available here): per cell the volume/level
inversion table at equally spaced volumes, per uv face depth/roughness/wet
fraction at equally spaced levels between ``uv_zmin`` and ``uv_zmax``.  The
core and the oracle both consume the same files, so table construction does
not affect parity.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import ncfile

G = 9.81


# --------------------------------------------------------------------------- DEMs
def fractal_surface(ny: int, nx: int, hurst: float, seed: int, device: str = "cpu"):
    """Zero-mean, unit-std fractal surface by spectral synthesis.

    Power spectral density ~ k^-(2H+2) (fractional Brownian surface with Hurst
    exponent H); random phases from a seeded generator.  Uses torch so that the
    multi-gigapixel DEMs of the large workloads are synthesised on the GPU.
    """
    import torch

    gen = torch.Generator(device=device).manual_seed(seed)
    ky = torch.fft.fftfreq(ny).to(torch.float32)
    kx = torch.fft.rfftfreq(nx).to(torch.float32)
    re = torch.randn(ny, nx // 2 + 1, generator=gen, dtype=torch.float32, device=device)
    im = torch.randn(ny, nx // 2 + 1, generator=gen, dtype=torch.float32, device=device)
    spec = torch.complex(re, im)
    del re, im
    k = torch.sqrt(ky.to(device)[:, None] ** 2 + kx.to(device)[None, :] ** 2)
    k[0, 0] = 1.0
    amp = k.pow(-(hurst + 1.0))
    amp[0, 0] = 0.0
    del k
    spec *= amp
    del amp
    z = torch.fft.irfft2(spec, s=(ny, nx))
    del spec
    z -= z.mean()
    z /= z.std().clamp_min(1e-12)
    return z


def coastal_dem(ny: int, nx: int, pixel: float, seed: int, zlo=-15.0, zhi=25.0,
                coast_x=30_000.0, noise_m=2.5, device: str = "cpu"):
    """Fractal coastal DEM: piecewise-linear trend (``zlo`` at x=0, 0 at
    ``coast_x``, ``zhi`` at the east edge) plus a Hurst-0.8 fractal, clipped to
    ``[zlo, zhi]``.  Returned as a float32 torch tensor ``(ny, nx)``."""
    import torch

    x = (torch.arange(nx, device=device, dtype=torch.float32) + 0.5) * pixel
    xe = nx * pixel
    trend = torch.where(x < coast_x, zlo * (1.0 - x / coast_x),
                        zhi * (x - coast_x) / max(xe - coast_x, 1.0))
    z = fractal_surface(ny, nx, 0.8, seed, device)
    z.mul_(noise_m).add_(trend[None, :])
    z.clamp_(zlo, zhi)
    return z


# ---------------------------------------------------------------- subgrid tables
def _cell_tables(z, area, nlev):
    """Volume/level tables for a batch of cells. z: (B, P) pixel elevations."""
    import torch

    s, _ = torch.sort(z.double(), dim=1)
    B, P = s.shape
    a = area / P
    zmin = s[:, 0]
    zmax = s[:, -1]
    csum = torch.cumsum(s, dim=1) - s  # exclusive prefix sum
    j = torch.arange(P, device=z.device, dtype=torch.float64)
    vj = a * (j[None, :] * s - csum)  # volume when the level reaches pixel j
    volmax = vj[:, -1]
    k = torch.arange(nlev, device=z.device, dtype=torch.float64)
    vt = volmax[:, None] * k[None, :] / (nlev - 1)
    idx = torch.searchsorted(vj.contiguous(), vt.contiguous(), right=True) - 1
    idx = idx.clamp(0, P - 1)
    sj = torch.gather(s, 1, idx)
    vjj = torch.gather(vj, 1, idx)
    lev = sj + (vt - vjj) / (a * (idx + 1).double())
    lev[:, 0] = zmin
    lev[:, -1] = zmax
    return zmin.float(), zmax.float(), volmax.float(), lev.float()


def _face_tables(z, mann, half, nlev):
    """uv-face tables for a batch of faces.

    z, mann: (B, P) pixels of the two half cells either side of the face;
    columns ``[:half]`` belong to the first cell, ``[half:]`` to the second.
    Returns zmin, zmax, havg(B,nlev), nrep(B,nlev), pwet(B,nlev), navg, ffit.
    """
    import torch

    zd = z.double()
    zmin = torch.maximum(zd[:, :half].min(dim=1).values, zd[:, half:].min(dim=1).values)
    zmax = zd.max(dim=1).values
    zmax = torch.maximum(zmax, zmin + 0.01)
    k = torch.arange(nlev, device=z.device, dtype=torch.float64)
    havg = torch.empty(z.shape[0], nlev, device=z.device, dtype=torch.float64)
    nrep = torch.empty_like(havg)
    pwet = torch.empty_like(havg)
    nd = mann.double()
    navg = nd.mean(dim=1)
    for i in range(nlev):
        zl = zmin + (zmax - zmin) * (i / (nlev - 1))
        h = (zl[:, None] - zd).clamp_min(0.0)
        ha = h.mean(dim=1)
        conv = (h.pow(5.0 / 3.0) / nd).mean(dim=1)
        nr = torch.where(conv > 0, ha.clamp_min(1e-12).pow(5.0 / 3.0) / conv.clamp_min(1e-30), navg)
        havg[:, i] = ha
        nrep[:, i] = nr
        pwet[:, i] = (h > 0).double().mean(dim=1)
    ffit = torch.ones_like(navg)
    return (zmin.float(), zmax.float(), havg.float(), nrep.float(), pwet.float(),
            navg.float(), ffit.float())


def build_subgrid_tables(dem, msk: np.ndarray, P: int, dx: float, dy: float, nlev: int = 10,
                         n_sea: float = 0.02, n_land: float = 0.04, rgh_lev: float = 0.0,
                         chunk_rows: int = 64) -> Dict[str, np.ndarray]:
    """Build the netCDF subgrid variables for a regular grid.

    ``dem``: torch tensor ``(nmax*P, mmax*P)`` (row 0 = south).  Pixel Manning
    n is ``n_sea`` below ``rgh_lev`` and ``n_land`` above.  Returns arrays in the
    reference's compacted order (active cells with n fastest; per cell its right
    u face then its upper v face, ``sfincs_domain.f90:727-1003``).
    """
    import torch

    nmax, mmax = msk.shape
    assert P % 2 == 0, "subpixel count per cell side must be even"
    h = P // 2
    act = msk > 0
    cz = {k: np.zeros((nmax, mmax), np.float32) for k in ("zmin", "zmax", "volmax")}
    clev = np.zeros((nmax, mmax, nlev), np.float32)
    fu = {}
    fv = {}
    area = dx * dy
    for r0 in range(0, nmax, chunk_rows):
        r1 = min(nmax, r0 + chunk_rows)
        blk = dem[r0 * P:r1 * P, :]  # rows of cells r0..r1-1
        nr = r1 - r0
        cells = blk.reshape(nr, P, mmax, P).permute(0, 2, 1, 3).reshape(nr * mmax, P * P)
        zmin, zmax, volmax, lev = _cell_tables(cells, area, nlev)
        cz["zmin"][r0:r1] = zmin.reshape(nr, mmax).cpu().numpy()
        cz["zmax"][r0:r1] = zmax.reshape(nr, mmax).cpu().numpy()
        cz["volmax"][r0:r1] = volmax.reshape(nr, mmax).cpu().numpy()
        clev[r0:r1] = lev.reshape(nr, mmax, nlev).cpu().numpy()
        del cells
        # u faces between (n,m) and (n,m+1): right half of cell m, left half of m+1
        if mmax > 1:
            sub = blk[:, h:h + (mmax - 1) * P]
            fz = sub.reshape(nr, P, mmax - 1, P).permute(0, 2, 1, 3)
            # order columns so that the first half belongs to the left cell
            fz = fz.reshape(nr * (mmax - 1), P, P)
            fz = torch.cat([fz[:, :, :h].reshape(-1, P * h), fz[:, :, h:].reshape(-1, P * h)], dim=1)
            mn = torch.where(fz < rgh_lev, n_sea, n_land).float()
            res = _face_tables(fz, mn, P * h, nlev)
            for key, val in zip(("zmin", "zmax", "havg", "nrep", "pwet", "navg", "ffit"), res):
                fu.setdefault(key, []).append(val.reshape(nr, mmax - 1, *val.shape[1:]).cpu().numpy())
    # v faces need rows spanning two cell rows: loop over cell rows
    for r0 in range(0, nmax - 1, chunk_rows):
        r1 = min(nmax - 1, r0 + chunk_rows)
        nr = r1 - r0
        blk = dem[r0 * P + h:r0 * P + h + nr * P, :]
        fz = blk.reshape(nr, P, mmax, P).permute(0, 2, 1, 3).reshape(nr * mmax, P, P)
        fz = torch.cat([fz[:, :h, :].reshape(-1, h * P), fz[:, h:, :].reshape(-1, h * P)], dim=1)
        mn = torch.where(fz < rgh_lev, n_sea, n_land).float()
        res = _face_tables(fz, mn, P * h, nlev)
        for key, val in zip(("zmin", "zmax", "havg", "nrep", "pwet", "navg", "ffit"), res):
            fv.setdefault(key, []).append(val.reshape(nr, mmax, *val.shape[1:]).cpu().numpy())
    U = {k: np.concatenate(v, axis=0) for k, v in fu.items()} if fu else {}
    V = {k: np.concatenate(v, axis=0) for k, v in fv.items()} if fv else {}

    # compacted order
    order = np.flatnonzero(act.ravel(order="F"))
    nn = order % nmax
    mm = order // nmax
    z_zmin = cz["zmin"][nn, mm]
    z_zmax = cz["zmax"][nn, mm]
    z_volmax = cz["volmax"][nn, mm]
    z_level = clev[nn, mm, :]
    faces = enumerate_faces(msk)
    out = {"z_zmin": z_zmin, "z_zmax": z_zmax, "z_volmax": z_volmax, "z_level": z_level}
    npuv = faces.shape[0]
    for key in ("zmin", "zmax", "havg", "nrep", "pwet", "navg", "ffit"):
        shape = (npuv,) + (U.get(key, V.get(key)).shape[2:])
        arr = np.zeros(shape, np.float32)
        iu = faces[:, 0] == 0
        iv = ~iu
        if iu.any():
            arr[iu] = U[key][faces[iu, 1], faces[iu, 2]]
        if iv.any():
            arr[iv] = V[key][faces[iv, 1], faces[iv, 2]]
        out["uv_" + key] = arr
    return out


def enumerate_faces(msk: np.ndarray) -> np.ndarray:
    """uv faces of a regular grid in the reference's order: loop over active
    cells with n fastest; per cell its right u face (if the right cell is
    active) then its upper v face (if the upper cell is active)
    (``sfincs_domain.f90:727-1003`` for a single-level mesh).
    Returns ``(npuv, 3)`` int64 rows ``(dir, n0, m0)`` (0-based cell of the face)."""
    nmax, mmax = msk.shape
    act = msk > 0
    has_u = np.zeros_like(act)
    has_u[:, :-1] = act[:, :-1] & act[:, 1:]
    has_v = np.zeros_like(act)
    has_v[:-1, :] = act[:-1, :] & act[1:, :]
    order = np.flatnonzero(act.ravel(order="F"))
    nn = order % nmax
    mm = order // nmax
    hu = has_u[nn, mm]
    hv = has_v[nn, mm]
    cnt = hu.astype(np.int64) + hv.astype(np.int64)
    first = np.cumsum(cnt) - cnt
    faces = np.empty((int(cnt.sum()), 3), np.int64)
    iu = first[hu]
    faces[iu, 0] = 0
    faces[iu, 1] = nn[hu]
    faces[iu, 2] = mm[hu]
    iv = first[hv] + hu[hv]
    faces[iv, 0] = 1
    faces[iv, 1] = nn[hv]
    faces[iv, 2] = mm[hv]
    return faces


def write_sbg(path: str, tables: Dict[str, np.ndarray]) -> None:
    """Write the subgrid netCDF variables read by ``sfincs_subgrid.F90:102-122``."""
    npz = tables["z_zmin"].shape[0]
    npuv = tables["uv_zmin"].shape[0]
    nlev = tables["z_level"].shape[1]
    ncfile.write(
        path,
        {"np": npz, "npuv": npuv, "levels": nlev},
        {
            "z_zmin": (("np",), tables["z_zmin"]),
            "z_zmax": (("np",), tables["z_zmax"]),
            "z_volmax": (("np",), tables["z_volmax"]),
            "z_level": (("np", "levels"), tables["z_level"]),
            "uv_zmin": (("npuv",), tables["uv_zmin"]),
            "uv_zmax": (("npuv",), tables["uv_zmax"]),
            "uv_havg": (("npuv", "levels"), tables["uv_havg"]),
            "uv_nrep": (("npuv", "levels"), tables["uv_nrep"]),
            "uv_pwet": (("npuv", "levels"), tables["uv_pwet"]),
            "uv_navg": (("npuv",), tables["uv_navg"]),
            "uv_ffit": (("npuv",), tables["uv_ffit"]),
        },
        {"source": "sfincs_b200 synthetic subgrid tables"},
    )


def write_meteo_grid(path: str, quantity: str, unit: str, x_ll: float, y_ll: float, dx: float, dy: float,
                     times_s, fields, ref: str = "2000-01-01 00:00:00") -> None:
    """Write a gridded meteo series in the ASCII equidistant-grid format the
    reference reads (amu / amv / amp / ampr files): header keys, then per time
    a ``TIME = <hours> hours since <ref>`` line and the field, top row first.
    ``fields`` is (nt, nrows, ncols) with row 0 at the bottom (y_ll)."""
    fields = np.asarray(fields, np.float64)
    nt, nrows, ncols = fields.shape
    with open(path, "w") as f:
        f.write("FileVersion      = 1.03\nfiletype         = meteo_on_equidistant_grid\n"
                f"NODATA_value     = -999.000\nn_cols           = {ncols}\nn_rows           = {nrows}\n"
                "grid_unit        = m\n"
                f"x_llcorner       = {x_ll:.4f}\ny_llcorner       = {y_ll:.4f}\ndx               = {dx:.4f}\n"
                f"dy               = {dy:.4f}\nn_quantity       = 1\nquantity1        = {quantity}\n"
                f"unit1            = {unit}\n")
        for it in range(nt):
            f.write(f"TIME = {times_s[it] / 3600.0:.6f} hours since {ref} +00:00\n")
            for row in fields[it][::-1]:
                f.write(" ".join(f"{v:.4f}" for v in row) + "\n")


def write_spiderweb(path: str, times_s, xe, ye, radius: float, vmag, vdir, pdrop, prcp=None,
                    ref: str = "2000-01-01 00:00:00") -> None:
    """Write a cyclone in the ASCII spiderweb format the reference reads
    (sfincs_spiderweb.f90:8-134): header keys, then per record a TIME line,
    the eye position, the eye pressure drop and ``nrows`` lines per quantity
    (wind speed, nautical from-direction, pressure drop, optionally rain in
    mm/h).  The quantity arrays are (nt, nrows, ncols): row i at radius
    i * radius / nrows, column j clockwise from north."""
    vmag = np.asarray(vmag, np.float64)
    nt, nrows, ncols = vmag.shape
    quants = [("wind_speed", "m s-1", vmag), ("wind_from_direction", "degree", vdir), ("p_drop", "Pa", pdrop)]
    if prcp is not None:
        quants.append(("precipitation", "mm/h", prcp))
    with open(path, "w") as f:
        f.write("FileVersion      = 1.03\nfiletype         = meteo_on_spiderweb_grid\n"
                f"NODATA_value     = -999.000\nn_cols           = {ncols}\nn_rows           = {nrows}\n"
                f"grid_unit        = m\nspw_radius       = {radius:.1f}\nspw_rad_unit     = m\n"
                f"n_quantity       = {len(quants)}\n")
        for k, (q, u, _) in enumerate(quants):
            f.write(f"quantity{k + 1}        = {q}\n")
        for k, (q, u, _) in enumerate(quants):
            f.write(f"unit{k + 1}            = {u}\n")
        for it in range(nt):
            f.write(f"TIME             = {times_s[it] / 3600.0:.6f} hours since {ref} +00:00\n")
            f.write(f"x_spw_eye        = {xe[it]:.2f}\ny_spw_eye        = {ye[it]:.2f}\n")
            f.write(f"p_drop_spw_eye   = {float(np.max(pdrop[it])):.1f}\n")
            for _, _, v in quants:
                for row in np.asarray(v, np.float64)[it]:
                    f.write(" ".join(f"{x:.3f}" for x in row) + "\n")


def cyclone(rng, nt: int, nrows: int, ncols: int, vmax: float = 45.0, rmax_frac: float = 0.2, dp: float = 4000.0,
            rain: float = 0.0):
    """Seeded polar fields of a synthetic cyclone (Rankine-like speed profile
    with noise, counter-clockwise from-directions with a 20 degree inflow,
    exponential pressure drop, rain peaking near the eye wall)."""
    r = (np.arange(1, nrows + 1) / nrows)[None, :, None]
    phi = (np.arange(ncols) * 360.0 / ncols)[None, None, :]
    prof = np.where(r < rmax_frac, r / rmax_frac, (rmax_frac / r) ** 0.6)
    vmag = vmax * prof * (1.0 + 0.1 * rng.standard_normal((nt, nrows, ncols)))
    vdir = np.mod(phi + 90.0 + 20.0 + 5.0 * rng.standard_normal((nt, nrows, ncols)), 360.0)
    pdrop = dp * np.exp(-r / (2 * rmax_frac)) * np.ones((nt, 1, ncols))
    out = dict(vmag=np.abs(vmag), vdir=vdir, pdrop=pdrop)
    if rain > 0:
        out["prcp"] = rain * np.exp(-((r - rmax_frac) / 0.2) ** 2) * (1 + 0.2 * np.abs(rng.standard_normal((nt, nrows, ncols))))
    return out


# ------------------------------------------------------------------ model files
@dataclass
class RegularModel:
    """A regular-grid SFINCS model written as the reference's input files."""

    msk: np.ndarray                      # (nmax, mmax) int8: 0 inactive, 1 regular, 2 bnd, 3 outflow, 6 Neumann
    dx: float
    dy: float
    zb: Optional[np.ndarray] = None      # (nmax, mmax) float32 (regular bathymetry)
    sbg: Optional[Dict[str, np.ndarray]] = None  # subgrid tables (compacted order)
    x0: float = 0.0
    y0: float = 0.0
    rotation: float = 0.0
    params: Dict[str, object] = field(default_factory=dict)
    bnd: Optional[np.ndarray] = None     # (nbnd, 2) x, y
    bzs: Optional[np.ndarray] = None     # (nt, 1+nbnd) t, zs...
    prcp: Optional[np.ndarray] = None    # (nt, 2) t, mm/h
    wnd: Optional[np.ndarray] = None     # (nt, 3) t, vmag, dir (nautical, from)
    qinf_field: Optional[np.ndarray] = None  # (nmax, mmax) mm/h for c2d infiltration
    src: Optional[np.ndarray] = None     # (nsrc, 2)
    dis: Optional[np.ndarray] = None     # (nt, 1+nsrc)
    thd: Optional[List[np.ndarray]] = None  # thin dams: polylines, each (npoints, 2) x, y
    weir: Optional[List[np.ndarray]] = None  # weirs: polylines, each (npoints, 4) x, y, crest level, Cd
    drn: Optional[List[Sequence[float]]] = None  # drainage: x_in, y_in, x_out, y_out, type, params...
    zsini_field: Optional[np.ndarray] = None  # (nmax, mmax) initial water level: binary inifile (real*4)
    cell_fields: Dict[str, np.ndarray] = field(default_factory=dict)  # keyword -> (nmax, mmax) binary real*4 file

    @property
    def nmax(self):
        return self.msk.shape[0]

    @property
    def mmax(self):
        return self.msk.shape[1]

    def compact(self, arr: np.ndarray) -> np.ndarray:
        return arr.ravel(order="F")[self.msk.ravel(order="F") > 0]

    def write(self, d: str) -> str:
        os.makedirs(d, exist_ok=True)
        act = self.msk.ravel(order="F") > 0
        ind = (np.flatnonzero(act) + 1).astype(np.int32)
        with open(os.path.join(d, "sfincs.ind"), "wb") as f:
            np.array([ind.size], np.int32).tofile(f)
            ind.tofile(f)
        self.compact(self.msk).astype(np.int8).tofile(os.path.join(d, "sfincs.msk"))
        inp: Dict[str, object] = {
            "mmax": self.mmax, "nmax": self.nmax, "dx": self.dx, "dy": self.dy,
            "x0": self.x0, "y0": self.y0, "rotation": self.rotation,
            "inputformat": "bin", "indexfile": "sfincs.ind", "mskfile": "sfincs.msk",
        }
        if self.zb is not None:
            self.compact(self.zb).astype(np.float32).tofile(os.path.join(d, "sfincs.dep"))
            inp["depfile"] = "sfincs.dep"
        if self.sbg is not None:
            write_sbg(os.path.join(d, "sfincs.sbg"), self.sbg)
            inp["sbgfile"] = "sfincs.sbg"
        if self.bnd is not None:
            np.savetxt(os.path.join(d, "sfincs.bnd"), self.bnd, fmt="%.8f" if self.params.get("crsgeo") else "%.4f")
            inp["bndfile"] = "sfincs.bnd"
        if self.bzs is not None:
            np.savetxt(os.path.join(d, "sfincs.bzs"), self.bzs, fmt="%.6f")
            inp["bzsfile"] = "sfincs.bzs"
        if self.prcp is not None:
            np.savetxt(os.path.join(d, "sfincs.prcp"), self.prcp, fmt="%.6f")
            inp["prcfile"] = "sfincs.prcp"
        if self.wnd is not None:
            np.savetxt(os.path.join(d, "sfincs.wnd"), self.wnd, fmt="%.6f")
            inp["wndfile"] = "sfincs.wnd"
        if self.qinf_field is not None:
            self.compact(self.qinf_field).astype(np.float32).tofile(os.path.join(d, "sfincs.qinf"))
            inp["qinffile"] = "sfincs.qinf"
        if self.src is not None:
            np.savetxt(os.path.join(d, "sfincs.src"), self.src, fmt="%.4f")
            np.savetxt(os.path.join(d, "sfincs.dis"), self.dis, fmt="%.6f")
            inp["srcfile"] = "sfincs.src"
            inp["disfile"] = "sfincs.dis"
        if self.thd:
            with open(os.path.join(d, "sfincs.thd"), "w") as f:
                for i, pl in enumerate(self.thd):
                    pl = np.asarray(pl, np.float64)
                    f.write(f"THD{i + 1:02d}\n{pl.shape[0]} 2\n")
                    for x, y in pl:
                        f.write(f"{x:.4f} {y:.4f}\n")
            inp["thdfile"] = "sfincs.thd"
        if self.weir:
            with open(os.path.join(d, "sfincs.weir"), "w") as f:
                for i, pl in enumerate(self.weir):
                    pl = np.asarray(pl, np.float64)
                    f.write(f"WEIR{i + 1:02d}\n{pl.shape[0]} 4\n")
                    for x, y, z, cd in pl:
                        f.write(f"{x:.4f} {y:.4f} {z:.4f} {cd:.4f}\n")
            inp["weirfile"] = "sfincs.weir"
        if self.drn:
            with open(os.path.join(d, "sfincs.drn"), "w") as f:
                for r in self.drn:
                    f.write(" ".join(str(int(v)) if k == 4 else f"{v:.4f}" for k, v in enumerate(r)) + "\n")
            inp["drnfile"] = "sfincs.drn"
        if self.zsini_field is not None:
            self.compact(self.zsini_field).astype(np.float32).tofile(os.path.join(d, "sfincs.ini"))
            inp["inifile"] = "sfincs.ini"
        for key, arr in self.cell_fields.items():
            self.compact(arr).astype(np.float32).tofile(os.path.join(d, f"sfincs.{key}"))
            inp[key] = f"sfincs.{key}"
        inp.update(self.params)
        with open(os.path.join(d, "sfincs.inp"), "w") as f:
            for k, v in inp.items():
                f.write(f"{k:<20} = {v}\n")
        return d


def _date(seconds: int) -> str:
    """``yyyymmdd HHMMSS`` for 2000-01-01 00:00:00 + seconds."""
    import datetime as _dt

    t = _dt.datetime(2000, 1, 1) + _dt.timedelta(seconds=int(seconds))
    return t.strftime("%Y%m%d %H%M%S")


def time_params(tstop_s: float) -> Dict[str, object]:
    return {"tref": _date(0), "tstart": _date(0), "tstop": _date(int(round(tstop_s)))}


# ------------------------------------------------------------------ named configs
def plain_regular(nmax=400, mmax=500, dx=50.0, seed=1, tstop=3600.0, nbumps=20) -> RegularModel:
    """Plain regular-grid workload (no subgrid, FP32): planar 1:100 beach from
    -10 m (west) to +10 m (east) over the grid length (25 km at 500x50 m) plus
    ``nbumps`` seeded Gaussian bumps (amplitude U(-2,2) m, sigma U(100,500) m);
    Manning 0.02 below 0 m, 0.04 above; west column water-level boundary with a
    1 m, 12.42 h sinusoidal tide; no advection, alpha=0.5, huthresh=0.01."""
    rng = np.random.default_rng(seed)
    L = mmax * dx
    x = (np.arange(mmax) + 0.5) * dx
    y = (np.arange(nmax) + 0.5) * dx
    X, Y = np.meshgrid(x, y)
    zb = -10.0 + 20.0 * X / L
    for _ in range(nbumps):
        a = rng.uniform(-2, 2)
        s = rng.uniform(100, 500)
        cx, cy = rng.uniform(0, L), rng.uniform(0, nmax * dx)
        zb += a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * s * s))
    msk = np.ones((nmax, mmax), np.int8)
    msk[:, 0] = 2
    tb = np.arange(0.0, tstop + 120.0, 60.0)
    bzs = np.stack([tb, np.sin(2 * np.pi * tb / 44712.0)], axis=1)
    params = dict(time_params(tstop))
    params.update({"alpha": 0.5, "huthresh": 0.01, "advection": 0, "manning_sea": 0.02,
                   "manning_land": 0.04, "rgh_lev_land": 0.0, "zsini": 0.0})
    return RegularModel(msk=msk, dx=dx, dy=dx, zb=zb.astype(np.float32), params=params,
                        bnd=np.array([[0.0, nmax * dx / 2]]), bzs=bzs)


def subgrid_regular(nmax=2000, mmax=2000, dx=100.0, P=20, seed=2, tstop=43200.0,
                    surge_peak=3.0, rain_mmh=40.0, rain_hours=3.0, nlev=10, coast_x=30_000.0,
                    device="cpu", t_peak=None, width_h=6.0) -> RegularModel:
    """Subgrid regular-grid workload: 10-level tables from a seeded fractal DEM
    (Hurst 0.8, relief -15..+25 m, coastline at ``coast_x``) at ``dx/P`` m pixels;
    a Gaussian surge hydrograph (peak ``surge_peak``; the "6 h width" is read as
    the full width at half maximum, sigma = 6 h / 2.355) on the west boundary
    and uniform rain ``rain_mmh`` for the first ``rain_hours``."""
    dem = coastal_dem(nmax * P, mmax * P, dx / P, seed, coast_x=coast_x, device=device)
    msk = np.ones((nmax, mmax), np.int8)
    msk[:, 0] = 2
    tables = build_subgrid_tables(dem, msk, P, dx, dx, nlev)
    del dem
    tp = tstop / 2 if t_peak is None else t_peak
    sig = width_h * 3600.0 / 2.355
    tb = np.arange(0.0, tstop + 1200.0, 600.0)
    bzs = np.stack([tb, surge_peak * np.exp(-0.5 * ((tb - tp) / sig) ** 2)], axis=1)
    tr = rain_hours * 3600.0
    prcp = np.array([[0.0, rain_mmh], [tr, rain_mmh], [tr + 1.0, 0.0], [tstop + 3600.0, 0.0]])
    params = dict(time_params(tstop))
    params.update({"alpha": 0.5, "zsini": 0.0})
    return RegularModel(msk=msk, dx=dx, dy=dx, sbg=tables, params=params,
                        bnd=np.array([[0.0, nmax * dx / 2]]), bzs=bzs, prcp=prcp)
