"""The oracle's gridded meteo (ASCII amu/amv/amp/ampr, sfincs_meteo.f90:
802-1442) against an independent numpy restatement of the reference's
bilinear interpolation, and its invariants."""
import numpy as np

from meteo_cases import add_meteo
from sfincs_b200 import synth

F = np.float32


def _plain(tmp_path, **params):
    m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
    m.params.update(params)
    return m


def _bilinear(g, fld, x, y):
    """update_ampr_data's interpolation of one record at one point (float32)."""
    nr, nc = g["nr"], g["nc"]
    dx, dy = F(float(f"{g['dx']:.4f}")), F(float(f"{g['dy']:.4f}"))
    x_ll, y_ll = F(float(f"{g['x_ll']:.4f}")), F(float(f"{g['y_ll']:.4f}"))
    yul = y_ll + F(nr - 1) * dy + F(0.5) * dy
    xll = x_ll + F(0.5) * dx
    iy = int((yul - y) / dy) + 1
    dj1 = (yul - F(iy - 1) * dy - y) / dy
    ix = int((x - xll) / dx) + 1
    di1 = (x - (xll + F(ix - 1) * dx)) / dx
    if iy <= 1 or iy >= nr or ix <= 0 or ix >= nc:
        return None
    f = [(F(1) - di1) * (F(1) - dj1), di1 * (F(1) - dj1), di1 * dj1, (F(1) - di1) * dj1]
    ind = [(iy, ix), (iy, ix + 1), (iy + 1, ix + 1), (iy + 1, ix)]
    v = F(0)
    for w, (r, c) in zip(f, ind):
        v = v + w * F(float(f"{fld[nr - r, c - 1]:.4f}"))  # file rows run from the top
    return v


def test_rain_field_matches_restated_interpolation(tmp_path):
    from oracle.oracle import Oracle

    m = _plain(tmp_path)
    d = m.write(str(tmp_path))
    g = add_meteo(d, m.mmax * m.dx, m.nmax * m.dy, wind=False, pres=False, rain=True)
    o = Oracle(d, "ref")
    o.update(-1000.0, 1)
    got = o.get("prcp")
    m_idx, n_idx = np.nonzero(m.msk.T > 0)  # compact order: n fastest
    xs = ((m_idx + 0.5) * m.dx).astype(F)
    ys = ((n_idx + 0.5) * m.dy).astype(F)
    inside = 0
    for k, (x, y) in enumerate(zip(xs, ys)):
        v = _bilinear(g, g["rain"][0], F(x), F(y))
        want = 0.0 if v is None else float(v / F(1000 * 3600))
        inside += v is not None
        assert abs(got[k] - want) <= 1e-6 * abs(want) + 1e-15, (k, got[k], want)
    assert inside > 0.8 * len(xs)


def test_pressure_and_wind_move_a_closed_basin(tmp_path):
    """Wind and a pressure gradient over a closed flat basin set the water in
    motion and keep its volume (FP64 accounting at the oracle's precision)."""
    from oracle.oracle import Oracle

    m = synth.plain_regular(nmax=16, mmax=20, dx=400.0, tstop=3600.0, nbumps=0)
    m.msk[:, 0] = 1
    m.bnd = m.bzs = None
    m.zb = np.full(m.msk.shape, -5.0, np.float32)
    d = m.write(str(tmp_path))
    add_meteo(d, m.mmax * m.dx, m.nmax * m.dy, rain=False)
    o = Oracle(d, "fp64")
    z0 = o.get("zs").sum()
    o.update(-1000.0, 200)
    zs = o.get("zs")
    assert np.abs(o.get("q")).max() > 1e-3
    assert abs(zs.sum() - z0) <= 1e-9 * zs.size
