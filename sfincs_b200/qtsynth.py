"""Synthetic quadtree meshes written as the reference's quadtree netCDF file.

A quadtree mesh here has ``nlev`` refinement levels over a level-1 grid of
``nmax1 x mmax1`` cells of ``dx1`` m; level L cells are ``dx1 / 2**(L-1)`` m.
Cells are refined by distance to a seeded random-walk coastline polyline and
the mesh is 2:1 balanced (side neighbours differ by at most one level).

The file carries what ``sfincs_quadtree.F90:295-440`` reads: per quadtree point
``n, m, level`` (1-based indices at the point's own level), the neighbour flags
``mu, md, nu, nd`` (0 same level, 1 two finer neighbours, -1 one coarser
neighbour) with neighbour point indices ``mu1, mu2, ...`` (1-based, 0 = none;
for two finer neighbours index 1 is the one with the lower n (right/left
faces) or lower m (upper/lower faces)), the bed level ``z``, the ``mask`` and
the global attributes ``x0, y0, dx, dy, rotation, nmax, mmax, nr_levels``.
Points are ordered by level, then by ``(m-1)*nmax_L + n`` (the order the
reference's binary search over ``quadtree_nm_indices`` requires).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from . import ncfile
from .synth import _cell_tables, _face_tables, time_params, write_sbg


def coastline_x(ny_px: int, pixel: float, seed: int, x_mean: float, amplitude: float) -> np.ndarray:
    """x of a random-walk coastline for every pixel row (seeded, smoothed,
    wandering within +-amplitude of x_mean)."""
    rng = np.random.default_rng(seed)
    nodes = max(8, ny_px // 64)
    steps = rng.normal(0.0, 1.0, nodes)
    walk = np.cumsum(steps)
    walk -= walk.mean()
    walk *= amplitude / max(np.abs(walk).max(), 1e-9)
    yn = np.linspace(0.0, ny_px * pixel, nodes)
    y = (np.arange(ny_px) + 0.5) * pixel
    return (x_mean + np.interp(y, yn, walk)).astype(np.float64)


def random_walk_polyline(seed: int, start, length: float, step: float, box) -> np.ndarray:
    """Seeded correlated 2-D random walk of total ``length`` m with segments of
    ``step`` m, reflected at the edges of ``box = (xmax, ymax)``."""
    rng = np.random.default_rng(seed)
    n = max(2, int(length / step))
    pts = np.empty((n + 1, 2))
    pts[0] = start
    ang = rng.uniform(0, 2 * np.pi)
    for i in range(n):
        ang += rng.normal(0.0, 0.35)
        p = pts[i] + step * np.array([np.cos(ang), np.sin(ang)])
        for k in (0, 1):
            if p[k] < 0 or p[k] > box[k]:
                p[k] = min(max(p[k], 0.0), box[k])
                ang = np.pi - ang if k == 0 else -ang
        pts[i + 1] = p
    return pts


def polyline_distance(pts: np.ndarray, ny: int, nx: int, px: float) -> np.ndarray:
    """Distance (m) from every pixel centre of an (ny, nx) raster of pixel size
    px to the polyline (rasterised at px/2 spacing, exact Euclidean transform)."""
    from scipy import ndimage

    seg = np.diff(pts, axis=0)
    lens = np.hypot(seg[:, 0], seg[:, 1])
    k = np.maximum(2, (lens / (0.5 * px)).astype(np.int64) + 1)
    sid = np.repeat(np.arange(seg.shape[0]), k)
    t = (np.arange(int(k.sum())) - np.repeat(np.cumsum(k) - k, k)) / np.repeat(k - 1, k)
    xs = ((pts[sid, 0] + t * seg[sid, 0]) / px).astype(np.int64)
    ys = ((pts[sid, 1] + t * seg[sid, 1]) / px).astype(np.int64)
    ok = (xs >= 0) & (xs < nx) & (ys >= 0) & (ys < ny)
    on = np.ones((ny, nx), bool)
    on[ys[ok], xs[ok]] = False
    return ndimage.distance_transform_edt(on) * px


def leaf_levels(nmax1: int, mmax1: int, dx1: float, nlev: int, xc_rows: np.ndarray, bands,
                dist: Optional[np.ndarray] = None) -> np.ndarray:
    """Leaf level of every finest-resolution pixel, refined by distance
    (``bands[k]``: distance within which cells are refined beyond level k+1)
    and then 2:1 balanced.  The distance is horizontal distance to the
    coastline x(row), or the given raster."""
    R = 1 << (nlev - 1)
    ny, nx = nmax1 * R, mmax1 * R
    px = dx1 / R
    if dist is None:
        x = (np.arange(nx) + 0.5) * px
        dist = np.abs(x[None, :] - xc_rows[:, None])
    target = np.ones((ny, nx), np.int8)
    for k, b in enumerate(bands[: nlev - 1]):
        target[dist < b] = k + 2
    lev = np.ones((ny, nx), np.int8)
    for L in range(1, nlev):
        b = R >> (L - 1)
        bm = target.reshape(ny // b, b, nx // b, b).max(axis=(1, 3))
        refine = np.repeat(np.repeat(bm > L, b, axis=0), b, axis=1)
        lev[refine & (lev == L)] = L + 1
    # 2:1 balance
    while True:
        nb = np.zeros_like(lev)
        nb[:, :-1] = np.maximum(nb[:, :-1], lev[:, 1:])
        nb[:, 1:] = np.maximum(nb[:, 1:], lev[:, :-1])
        nb[:-1, :] = np.maximum(nb[:-1, :], lev[1:, :])
        nb[1:, :] = np.maximum(nb[1:, :], lev[:-1, :])
        bad = nb > lev + 1
        if not bad.any():
            break
        for L in range(1, nlev):
            b = R >> (L - 1)
            m = (bad & (lev == L)).reshape(ny // b, b, nx // b, b).any(axis=(1, 3))
            if m.any():
                up = np.repeat(np.repeat(m, b, axis=0), b, axis=1)
                lev[up & (lev == L)] = L + 1
    return lev


@dataclass
class QuadtreeMesh:
    nmax1: int
    mmax1: int
    dx1: float
    nlev: int
    level: np.ndarray          # [npq] int32
    n: np.ndarray              # [npq] int32, 1-based at the point's level
    m: np.ndarray
    nbr: Dict[str, np.ndarray]  # flags mu, md, nu, nd and indices mu1, mu2, ... (1-based, 0 = none)
    x0: float = 0.0
    y0: float = 0.0

    @property
    def npq(self) -> int:
        return int(self.level.size)

    def size(self, i) -> float:
        return self.dx1 / (1 << (int(self.level[i]) - 1))


def build_mesh(lev: np.ndarray, nmax1: int, mmax1: int, dx1: float, nlev: int) -> QuadtreeMesh:
    R = 1 << (nlev - 1)
    levels, ns, ms = [], [], []
    for L in range(1, nlev + 1):
        b = R >> (L - 1)
        blk = lev[::b, ::b] == L  # the block's first pixel; leaves are uniform blocks
        # a level-L leaf: every pixel of the block has level L
        full = (lev.reshape(lev.shape[0] // b, b, lev.shape[1] // b, b) == L).all(axis=(1, 3))
        ii, jj = np.nonzero(blk & full)
        levels.append(np.full(ii.size, L, np.int32))
        ns.append((ii + 1).astype(np.int32))
        ms.append((jj + 1).astype(np.int32))
    level = np.concatenate(levels)
    n = np.concatenate(ns)
    m = np.concatenate(ms)
    # order: level, then (m-1)*nmax_L + n
    nmaxL = nmax1 << (level.astype(np.int64) - 1)
    key = level.astype(np.int64) * (1 << 40) + (m.astype(np.int64) - 1) * nmaxL + n
    order = np.argsort(key, kind="stable")
    level, n, m = level[order], n[order], m[order]
    npq = level.size
    # per-level index grids (1-based point index, 0 = no leaf at that level)
    grids = {}
    for L in range(1, nlev + 1):
        g = np.zeros((nmax1 << (L - 1), mmax1 << (L - 1)), np.int32)
        sel = np.nonzero(level == L)[0]
        g[n[sel] - 1, m[sel] - 1] = sel + 1
        grids[L] = g

    def at(L, nn, mm):
        """Point index at level L of 1-based (nn, mm) arrays, 0 outside / none."""
        out = np.zeros(nn.shape, np.int32)
        if L < 1 or L > nlev:
            return out
        g = grids[L]
        ok = (nn >= 1) & (mm >= 1) & (nn <= g.shape[0]) & (mm <= g.shape[1])
        out[ok] = g[nn[ok] - 1, mm[ok] - 1]
        return out

    nbr = {}
    for side in ("mu", "md", "nu", "nd"):
        flag = np.zeros(npq, np.int32)
        i1 = np.zeros(npq, np.int32)
        i2 = np.zeros(npq, np.int32)
        for L in range(1, nlev + 1):
            sel = np.nonzero(level == L)[0]
            if sel.size == 0:
                continue
            nn, mm = n[sel].astype(np.int64), m[sel].astype(np.int64)
            if side == "mu":
                same = at(L, nn, mm + 1)
                coarse = at(L - 1, (nn + 1) // 2, (mm + 2) // 2)
                f1, f2 = at(L + 1, 2 * nn - 1, 2 * mm + 1), at(L + 1, 2 * nn, 2 * mm + 1)
            elif side == "md":
                same = at(L, nn, mm - 1)
                coarse = at(L - 1, (nn + 1) // 2, mm // 2)
                f1, f2 = at(L + 1, 2 * nn - 1, 2 * mm - 2), at(L + 1, 2 * nn, 2 * mm - 2)
            elif side == "nu":
                same = at(L, nn + 1, mm)
                coarse = at(L - 1, (nn + 2) // 2, (mm + 1) // 2)
                f1, f2 = at(L + 1, 2 * nn + 1, 2 * mm - 1), at(L + 1, 2 * nn + 1, 2 * mm)
            else:
                same = at(L, nn - 1, mm)
                coarse = at(L - 1, nn // 2, (mm + 1) // 2)
                f1, f2 = at(L + 1, 2 * nn - 2, 2 * mm - 1), at(L + 1, 2 * nn - 2, 2 * mm)
            fl = np.zeros(sel.size, np.int32)
            a = np.zeros(sel.size, np.int32)
            b = np.zeros(sel.size, np.int32)
            s = same > 0
            a[s] = same[s]
            c = (~s) & (coarse > 0)
            fl[c] = -1
            a[c] = coarse[c]
            f = (~s) & (~c) & ((f1 > 0) | (f2 > 0))
            fl[f] = 1
            a[f] = f1[f]
            b[f] = f2[f]
            flag[sel], i1[sel], i2[sel] = fl, a, b
        nbr[side] = flag
        nbr[side + "1"] = i1
        nbr[side + "2"] = i2
    return QuadtreeMesh(nmax1, mmax1, dx1, nlev, level, n, m, nbr)


def quadtree_faces(mesh: QuadtreeMesh, active: Optional[np.ndarray] = None):
    """Faces in the quadtree file's own order (``sfincs_subgrid.F90:163-231``):
    per point, its right face(s) then its upper face(s).  Returns rows
    ``(dir, point_a, point_b)`` (0-based points, a left/below of b)."""
    rows = []
    nb = mesh.nbr
    for ip in range(mesh.npq):
        for side, d in (("mu", 0), ("nu", 1)):
            if nb[side][ip] < 1:
                if nb[side + "1"][ip] > 0:
                    rows.append((d, ip, nb[side + "1"][ip] - 1))
            else:
                if nb[side + "1"][ip] > 0:
                    rows.append((d, ip, nb[side + "1"][ip] - 1))
                if nb[side + "2"][ip] > 0:
                    rows.append((d, ip, nb[side + "2"][ip] - 1))
    return np.array(rows, np.int64).reshape(-1, 3)


def _pix_block(dem, mesh: QuadtreeMesh, ip: int, R: int, P: int):
    """DEM pixels of point ip (rows n, cols m) at P pixels per finest cell."""
    L = int(mesh.level[ip])
    b = (R >> (L - 1)) * P
    r0 = (int(mesh.n[ip]) - 1) * b
    c0 = (int(mesh.m[ip]) - 1) * b
    return dem[r0:r0 + b, c0:c0 + b]


def build_quadtree_tables(dem, mesh: QuadtreeMesh, P: int, nlev_tab: int = 10, n_sea: float = 0.02,
                          n_land: float = 0.04, rgh_lev: float = 0.0) -> Dict[str, np.ndarray]:
    """Subgrid tables of every quadtree point and face (file order).  ``dem``
    is a torch tensor at ``P`` pixels per finest cell.  A face uses the pixels
    of the half cell on either side across the width of the smaller cell."""
    import torch

    R = 1 << (mesh.nlev - 1)
    npq = mesh.npq
    z_zmin = np.zeros(npq, np.float32)
    z_zmax = np.zeros(npq, np.float32)
    z_volmax = np.zeros(npq, np.float32)
    z_level = np.zeros((npq, nlev_tab), np.float32)
    for L in range(1, mesh.nlev + 1):
        sel = np.nonzero(mesh.level == L)[0]
        if sel.size == 0:
            continue
        b = (R >> (L - 1)) * P
        area = (mesh.dx1 / (1 << (L - 1))) ** 2
        rows = torch.as_tensor((mesh.n[sel] - 1).astype(np.int64) * b, device=dem.device)
        cols = torch.as_tensor((mesh.m[sel] - 1).astype(np.int64) * b, device=dem.device)
        off = torch.arange(b, device=dem.device)
        for s0 in range(0, sel.size, 4096):
            rr = rows[s0:s0 + 4096, None, None] + off[None, :, None]
            cc = cols[s0:s0 + 4096, None, None] + off[None, None, :]
            pix = dem[rr, cc].reshape(rr.shape[0], b * b)
            zmin, zmax, volmax, lev = _cell_tables(pix, area, nlev_tab)
            k = sel[s0:s0 + 4096]
            z_zmin[k] = zmin.cpu().numpy()
            z_zmax[k] = zmax.cpu().numpy()
            z_volmax[k] = volmax.cpu().numpy()
            z_level[k] = lev.cpu().numpy()
    faces = quadtree_faces(mesh)
    nf = faces.shape[0]
    out = {"z_zmin": z_zmin, "z_zmax": z_zmax, "z_volmax": z_volmax, "z_level": z_level}
    U = {k: np.zeros(nf, np.float32) for k in ("zmin", "zmax", "navg", "ffit")}
    for k in ("havg", "nrep", "pwet"):
        U[k] = np.zeros((nf, nlev_tab), np.float32)
    # group faces by (dir, width in pixels) so each batch has one shape
    la = mesh.level[faces[:, 1]]
    lb = mesh.level[faces[:, 2]]
    lf = np.maximum(la, lb)  # the smaller cell sets the face width
    for d in (0, 1):
        for L in range(1, mesh.nlev + 1):
            sel_all = np.nonzero((faces[:, 0] == d) & (lf == L))[0]
            for c0 in range(0, sel_all.size, 8192):
                _face_batch(dem, mesh, faces, la, lb, sel_all[c0:c0 + 8192], d, L, R, P, nlev_tab, n_sea, n_land,
                            rgh_lev, U)
    for key, val in U.items():
        out["uv_" + key] = val
    return out


def _face_batch(dem, mesh, faces, la, lb, sel, d, L, R, P, nlev_tab, n_sea, n_land, rgh_lev, U):
    import torch

    if True:
        if True:
            w = (R >> (L - 1)) * P      # face width in pixels
            h = w // 2                   # half-cell depth on each side
            a = faces[sel, 1]
            bb = faces[sel, 2]
            # face position: along the shared edge, the smaller cell's extent
            small = np.where(la[sel] >= lb[sel], a, bb)
            if d == 0:
                # vertical edge at the right side of a (= left side of b)
                xe = mesh.m[bb].astype(np.int64) - 1
                xe = xe * ((R >> (mesh.level[bb] - 1)) * P)
                y0 = (mesh.n[small].astype(np.int64) - 1) * ((R >> (mesh.level[small] - 1)) * P)
                rr = torch.as_tensor(y0, device=dem.device)[:, None, None] + torch.arange(w, device=dem.device)[None, :, None]
                cc = torch.as_tensor(xe - h, device=dem.device)[:, None, None] + torch.arange(2 * h, device=dem.device)[None, None, :]
                pix = dem[rr, cc]                       # (B, w, 2h): left half then right half along columns
                fz = torch.cat([pix[:, :, :h].reshape(-1, w * h), pix[:, :, h:].reshape(-1, w * h)], dim=1)
            else:
                ye = (mesh.n[bb].astype(np.int64) - 1) * ((R >> (mesh.level[bb] - 1)) * P)
                x0 = (mesh.m[small].astype(np.int64) - 1) * ((R >> (mesh.level[small] - 1)) * P)
                rr = torch.as_tensor(ye - h, device=dem.device)[:, None, None] + torch.arange(2 * h, device=dem.device)[None, :, None]
                cc = torch.as_tensor(x0, device=dem.device)[:, None, None] + torch.arange(w, device=dem.device)[None, None, :]
                pix = dem[rr, cc]                       # (B, 2h, w): lower half then upper half along rows
                fz = torch.cat([pix[:, :h, :].reshape(-1, h * w), pix[:, h:, :].reshape(-1, h * w)], dim=1)
            mn = torch.where(fz < rgh_lev, n_sea, n_land).float()
            res = _face_tables(fz, mn, w * h, nlev_tab)
            for key, val in zip(("zmin", "zmax", "havg", "nrep", "pwet", "navg", "ffit"), res):
                U[key][sel] = val.cpu().numpy()


@dataclass
class QuadtreeModel:
    """A quadtree SFINCS model written as the reference's input files."""

    mesh: QuadtreeMesh
    mask: np.ndarray                    # [npq] int8 (0 inactive, 1 active, 2 water-level boundary)
    z: np.ndarray                       # [npq] float32 bed level (used when there is no subgrid)
    sbg: Optional[Dict[str, np.ndarray]] = None
    rotation: float = 0.0
    params: Dict[str, object] = field(default_factory=dict)
    bnd: Optional[np.ndarray] = None
    bzs: Optional[np.ndarray] = None
    prcp: Optional[np.ndarray] = None
    wnd: Optional[np.ndarray] = None

    def write(self, d: str) -> str:
        os.makedirs(d, exist_ok=True)
        me = self.mesh
        v = {"n": (("mesh2d_nFaces",), me.n.astype(np.int32)),
             "m": (("mesh2d_nFaces",), me.m.astype(np.int32)),
             "level": (("mesh2d_nFaces",), me.level.astype(np.int32))}
        for k in ("md", "md1", "md2", "mu", "mu1", "mu2", "nd", "nd1", "nd2", "nu", "nu1", "nu2"):
            v[k] = (("mesh2d_nFaces",), me.nbr[k].astype(np.int32))
        v["z"] = (("mesh2d_nFaces",), self.z.astype(np.float32))
        v["mask"] = (("mesh2d_nFaces",), self.mask.astype(np.int8))
        ncfile.write(os.path.join(d, "sfincs.qtr.nc"), {"mesh2d_nFaces": me.npq}, v,
                     {"x0": np.float64(me.x0), "y0": np.float64(me.y0), "dx": np.float64(me.dx1),
                      "dy": np.float64(me.dx1), "rotation": np.float64(self.rotation),
                      "nmax": np.int32(me.nmax1), "mmax": np.int32(me.mmax1), "nr_levels": np.int32(me.nlev)})
        inp: Dict[str, object] = {"qtrfile": "sfincs.qtr.nc", "inputformat": "bin"}
        if self.sbg is not None:
            write_sbg(os.path.join(d, "sfincs.sbg"), self.sbg)
            inp["sbgfile"] = "sfincs.sbg"
        if self.bnd is not None:
            np.savetxt(os.path.join(d, "sfincs.bnd"), self.bnd, fmt="%.4f")
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
        inp.update(self.params)
        with open(os.path.join(d, "sfincs.inp"), "w") as f:
            for k, val in inp.items():
                f.write(f"{k:<20} = {val}\n")
        return d


def quadtree_coastal(nmax1=40, mmax1=60, dx1=400.0, nlev=4, bands=(2000.0, 1000.0, 500.0), P=4, seed=3,
                     tstop=21600.0, subgrid=True, tide_amp=1.5, tide_period=44712.0, wind_speed=30.0,
                     coast_frac=0.4, coast_wander=0.1, device="cpu", nlev_tab=10,
                     advection=1, viscosity=1, walk_km: float = 0.0) -> QuadtreeModel:
    """Quadtree coastal model: ``nlev`` levels from ``dx1`` down, refined within
    ``bands`` of a random-walk coastline (sea to the west), a fractal DEM at
    ``P`` pixels per finest cell (relief -15..+25 m), a water-level boundary
    on the west edge with a sinusoidal tide, and a uniform onshore wind
    (from the west) of ``wind_speed`` m/s.  With ``walk_km`` > 0 the
    refinement follows a seeded 2-D random-walk polyline of that length
    starting on the coast (distance-banded as for the coastline) instead of
    the coastline itself."""
    import torch

    R = 1 << (nlev - 1)
    ny_px = nmax1 * R * P
    nx_px = mmax1 * R * P
    pixel = dx1 / R / P
    xw = mmax1 * dx1
    xc = coastline_x(ny_px, pixel, seed, coast_frac * xw, coast_wander * xw)
    # leaf levels from the coastline at the finest cell rows
    xc_rows = xc.reshape(nmax1 * R, P).mean(axis=1)
    dist = None
    if walk_km > 0:
        ny_c, nx_c = nmax1 * R, mmax1 * R
        pts = random_walk_polyline(seed + 1, (float(xc_rows[ny_c // 2]), ny_c * dx1 / R / 2), walk_km * 1000.0,
                                   200.0, (nx_c * dx1 / R, ny_c * dx1 / R))
        dist = polyline_distance(pts, ny_c, nx_c, dx1 / R)
    lev = leaf_levels(nmax1, mmax1, dx1, nlev, xc_rows, bands, dist)
    del dist
    mesh = build_mesh(lev, nmax1, mmax1, dx1, nlev)
    # DEM: trend relative to the local coastline plus a fractal
    from .synth import fractal_surface

    x = (torch.arange(nx_px, device=device, dtype=torch.float32) + 0.5) * pixel
    xcr = torch.as_tensor(xc, device=device, dtype=torch.float32)
    dxr = x[None, :] - xcr[:, None]
    zlo, zhi = -15.0, 25.0
    trend = torch.where(dxr < 0, zlo * torch.clamp(-dxr / xcr.clamp_min(1.0)[:, None], max=1.0),
                        zhi * torch.clamp(dxr / (xw - xcr).clamp_min(1.0)[:, None], max=1.0))
    dem = fractal_surface(ny_px, nx_px, 0.8, seed, device) * 2.5 + trend
    dem.clamp_(zlo, zhi)
    del trend, dxr
    # bed level per point: mean of its pixels
    z = np.zeros(mesh.npq, np.float32)
    for L in range(1, nlev + 1):
        sel = np.nonzero(mesh.level == L)[0]
        b = (R >> (L - 1)) * P
        blk = dem.reshape(ny_px // b, b, nx_px // b, b).mean(dim=(1, 3)).cpu().numpy()
        z[sel] = blk[mesh.n[sel] - 1, mesh.m[sel] - 1]
    mask = np.ones(mesh.npq, np.int8)
    mask[mesh.m == 1] = 2  # west edge (m = 1 at every level)
    sbg = build_quadtree_tables(dem, mesh, P, nlev_tab) if subgrid else None
    del dem
    t = np.arange(0.0, tstop + 1200.0, 600.0)
    bzs = np.stack([t, tide_amp * np.sin(2.0 * np.pi * t / tide_period)], axis=1)
    wnd = np.array([[0.0, wind_speed, 270.0], [tstop + 3600.0, wind_speed, 270.0]])
    params = dict(time_params(tstop))
    params.update({"alpha": 0.5, "zsini": 0.0, "advection": advection, "viscosity": viscosity})
    return QuadtreeModel(mesh=mesh, mask=mask, z=z, sbg=sbg, params=params,
                         bnd=np.array([[0.0, nmax1 * dx1 / 2]]), bzs=bzs, wnd=wnd)
