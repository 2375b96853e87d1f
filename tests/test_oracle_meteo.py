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


def test_core_arctangent_is_accurate():
    """The core's IEEE-only arctangent stays within 2 ulp of atan2 in float64,
    over all four quadrants, both octants and the axes."""
    import ctypes

    from oracle.oracle import lib

    f = lib().oracle_core_atan2
    f.restype = ctypes.c_float
    f.argtypes = [ctypes.c_float, ctypes.c_float]
    rng = np.random.default_rng(7)
    ys = np.concatenate([rng.standard_normal(4000) * 10.0 ** rng.integers(-3, 5, 4000), [0.0, 0.0, 1.0, -1.0, 3.0]])
    xs = np.concatenate([rng.standard_normal(4000) * 10.0 ** rng.integers(-3, 5, 4000), [1.0, 0.0, 0.0, 0.0, 3.0]])
    worst = 0.0
    for y, x in zip(ys.astype(F), xs.astype(F)):
        got = F(f(float(y), float(x)))
        want = np.arctan2(np.float64(y), np.float64(x))
        if want == 0.0:
            assert got == 0.0
            continue
        ulp = float(np.spacing(F(abs(want))))
        worst = max(worst, abs(float(got) - want) / ulp)
    assert worst <= 2.0, worst


def _spw_expected(w, gapres, x, y, meteo_t, cdval):
    """update_spiderweb_data at one end of a window for one point (float32,
    numpy's arctangent), over no background: (tau_u, tau_v, patm, prcp)."""
    times = w["times"].astype(F)
    nt, nr, nc = w["vmag"].shape
    tf = F(meteo_t)
    if tf < times[0]:
        i0 = i1 = 0
        tw, spin = F(1), max(F(1) - (times[0] - tf) / F(21600), F(0))
    elif tf > times[-1]:
        i0 = i1 = nt - 1
        tw, spin = F(1), max(F(1) - (tf - times[-1]) / F(21600), F(0))
    else:
        i0 = int(np.nonzero(times <= tf)[0][-1])
        i1 = min(i0 + 1, nt - 1)
        tw, spin = (tf - times[i0]) / max(times[i1] - times[i0], F(1e-6)), F(1)
    pi = F(3.14159)
    rd = lambda v: np.array([[[float(f"{e:.3f}") for e in row] for row in rec] for rec in v], F)  # noqa: E731
    ang = pi * (F(270) - rd(w["vdir"])) / F(180)
    wu = rd(w["vmag"]) * np.cos(ang)
    wv = rd(w["vmag"]) * np.sin(ang)
    pabs = F(gapres) - rd(w["pdrop"])
    pr = rd(w["prcp"])
    xe = F(float(f"{w['xe'][i0]:.2f}")) * (F(1) - tw) + F(float(f"{w['xe'][i1]:.2f}")) * tw
    ye = F(float(f"{w['ye'][i0]:.2f}")) * (F(1) - tw) + F(float(f"{w['ye'][i1]:.2f}")) * tw
    R = F(float(f"{w['radius']:.1f}"))
    drad, dphi = R / F(nr), F(2) * pi / F(nc)
    dxe, dye = F(x) - xe, F(y) - ye
    dst = np.sqrt(dxe * dxe + dye * dye)
    if dst > R:
        return 0.0, 0.0, gapres, 0.0
    idst = max(int(dst / drad), 1)
    if idst + 1 > nr:
        return 0.0, 0.0, gapres, 0.0
    dj1 = max((dst - drad * F(idst)) / drad, F(0))
    phi = F(0.5) * pi - np.arctan2(dye, dxe)
    if phi < 0:
        phi = phi + F(2) * pi
    iphi = min(int(phi / dphi) + 1, nc)
    di1 = (phi - dphi * F(iphi - 1)) / dphi
    ind = [(idst, iphi), (idst, iphi % nc + 1), (idst + 1, iphi % nc + 1), (idst + 1, iphi)]
    f = [(F(1) - di1) * (F(1) - dj1), di1 * (F(1) - dj1), di1 * dj1, (F(1) - di1) * dj1]
    v = lambda a, r, c: a[i0, r - 1, c - 1] * (F(1) - tw) + a[i1, r - 1, c - 1] * tw  # noqa: E731
    wup = sum(fk * v(wu, r, c) for fk, (r, c) in zip(f, ind))
    wvp = sum(fk * v(wv, r, c) for fk, (r, c) in zip(f, ind))
    pcp = sum(fk * v(pabs, r, c) for fk, (r, c) in zip(f, ind))
    prp = sum(fk * v(pr, r, c) for fk, (r, c) in zip(f, ind))
    vmag = np.sqrt(wup * wup + wvp * wvp)
    cd = cdval[min(int(vmag * F(10)) + 1, 1000) - 1]
    merge = F(1)
    if dst > F(0.5) * R:
        merge = (F(1) / (F(1) - F(0.5))) * (R - dst) / R
    merge = merge * spin
    rho = F(1.25) * cd / F(1024)
    return (float(merge * vmag * wup * rho), float(merge * vmag * wvp * rho),
            float((F(1) - merge) * F(gapres) + merge * pcp), float(merge * prp / F(3600000)))


def _cdval():
    """The default drag table (sfincs_meteo.f90:314-327), float32."""
    out = np.zeros(1000, F)
    for iw in range(1, 1001):
        wnd = F(iw) * F(0.1)
        if wnd < F(28):
            out[iw - 1] = F(0.0010) + (wnd - F(0)) * (F(0.0025) - F(0.0010)) / F(28)
        elif wnd < F(50):
            out[iw - 1] = F(0.0025) + (wnd - F(28)) * (F(0.0015) - F(0.0025)) / F(22)
        else:
            out[iw - 1] = F(0.0015)
    return out


def test_spiderweb_window_matches_restatement(tmp_path):
    """The oracle's spiderweb window fields (wind stress, pressure, rain at
    both ends of the first two windows) against a numpy float32 restatement of
    update_spiderweb_data (sfincs_meteo.f90:450-800)."""
    from meteo_cases import add_spiderweb
    from oracle.oracle import Oracle

    m = _plain(tmp_path)
    d = m.write(str(tmp_path))
    w = add_spiderweb(d, m.mmax * m.dx, m.nmax * m.dy)
    o = Oracle(d, "ref")
    m_idx, n_idx = np.nonzero(m.msk.T > 0)
    xs = ((m_idx + 0.5) * m.dx).astype(F)
    ys = ((n_idx + 0.5) * m.dy).astype(F)
    cd = _cdval()
    checked = 0
    for window in range(2):
        o.update(-1000.0, 1)
        while o.scalars()["t"] < 600.0 * window:
            o.update(-1000.0, 1)
        got = {k: o.get(k) for k in ("tauwu0", "tauwv0", "patm0", "prcp0", "tauwu1", "patm1", "prcp1")}
        t0 = 600.0 * window
        for k in range(0, len(xs), 7):
            for end, tt in ((0, t0), (1, t0 + 600.0)):
                tu, tv, p, pr = _spw_expected(w, 101200.0, xs[k], ys[k], tt, cd)
                sfx = str(end)
                assert abs(got["tauwu" + sfx][k] - tu) <= 1e-5 * abs(tu) + 1e-9, (window, k, end)
                assert abs(got["patm" + sfx][k] - p) <= 1e-6 * p, (window, k, end)
                assert abs(got["prcp" + sfx][k] - pr) <= 1e-5 * abs(pr) + 1e-14, (window, k, end)
                if end == 0:
                    assert abs(got["tauwv0"][k] - tv) <= 1e-5 * abs(tv) + 1e-9
                checked += tu != 0.0
    assert checked > 20


def test_spiderweb_cyclone_moves_a_closed_basin(tmp_path):
    """A spiderweb cyclone over a closed flat basin sets the water in motion,
    its pressure drop raises the level under the eye, and the volume holds
    (rain off)."""
    from meteo_cases import add_spiderweb
    from oracle.oracle import Oracle

    m = synth.plain_regular(nmax=16, mmax=20, dx=400.0, tstop=3600.0, nbumps=0)
    m.msk[:, 0] = 1
    m.bnd = m.bzs = None
    m.zb = np.full(m.msk.shape, -5.0, np.float32)
    d = m.write(str(tmp_path))
    add_spiderweb(d, m.mmax * m.dx, m.nmax * m.dy, rain=0.0)
    o = Oracle(d, "fp64")
    z0 = o.get("zs").sum()
    o.update(-1000.0, 300)
    zs = o.get("zs")
    assert np.abs(o.get("q")).max() > 1e-3
    assert abs(zs.sum() - z0) <= 1e-9 * zs.size
