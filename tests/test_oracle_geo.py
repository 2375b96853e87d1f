"""The oracle on geographic grids (crsgeo = 1; sfincs_domain.f90:1403-1473,
sfincs_momentum.f90:205-234, sfincs_continuity.f90:94-147, 350-361, 458-470):
cell widths and areas against a numpy restatement, lake at rest, volume
balance with rain on a closed basin, and agreement with the projected grid
of the same spacing at the equator."""
import math

import numpy as np

from geo_cases import R, geographic
from sfincs_b200 import synth

F = np.float32


def _basin(tmp_path, lat0, rain=True):
    m = synth.plain_regular(nmax=14, mmax=18, dx=300.0, tstop=1800.0, seed=4, nbumps=3)
    m.msk[:, 0] = 1
    m.bnd = m.bzs = None
    m.params.update(advection=1, coriolis=1)
    if rain:
        m.prcp = np.array([[0.0, 30.0], [1800.0, 30.0]])
    geographic(m, lat0=lat0)
    return m.write(str(tmp_path)), m


def test_cell_widths_and_areas(tmp_path):
    from oracle.oracle import Oracle

    d, m = _basin(tmp_path, 52.0)
    o = Oracle(d, "ref")
    mi, ni = np.nonzero(m.msk.T > 0)
    dx, dy = F(m.dx), F(m.dy)
    yz = F(m.y0) + (F(1.0) * (ni.astype(F) + F(0.5))) * dy  # z_yz without rotation
    pi = F(3.14159)
    dxm = dx * F(R) * np.cos(yz * pi / F(180)).astype(F)
    area = dxm * (F(R) * dy)
    n = len(mi)
    assert np.allclose(o.get("dxm", n), dxm, rtol=2e-7)
    assert np.allclose(o.get("cell_area_m2", n), area, rtol=3e-7)
    # widths shrink towards the pole: the northern row is narrower than the southern one
    assert dxm[ni == ni.max()].max() < dxm[ni == 0].min()


def test_lake_at_rest_is_bitwise_still(tmp_path):
    from oracle.oracle import Oracle

    d, m = _basin(tmp_path, 40.0, rain=False)
    with open(d + "/sfincs.inp", "a") as f:
        f.write(f"{'zsini':<20} = 5.0\n")
    o = Oracle(d, "f32")
    z0 = o.get("zs").copy()
    o.update(-1000.0, 60)
    assert np.array_equal(o.get("zs"), z0)
    assert np.all(o.get("q") == 0.0)


def test_rain_volume_balance_on_a_closed_basin(tmp_path):
    from oracle.oracle import Oracle

    d, m = _basin(tmp_path, 40.0)
    o = Oracle(d, "fp64")
    n = int(o.scalars()["np"])
    area = o.get("cell_area_m2", n)
    zb = o.get("zb")
    v0 = float(((o.get("zs") - zb) * area).sum())
    o.update(-1000.0, 200)
    s = o.scalars()
    v1 = float(((o.get("zs") - zb) * area).sum())
    rain = 30.0 / 3.6e6 * (s["t"] - s["t0"]) * area.sum()
    assert abs((v1 - v0) - rain) <= 1e-6 * rain, (v1 - v0, rain)
    assert np.abs(o.get("q")).max() > 1e-4  # Coriolis and the bed moved the water


def test_equator_matches_the_projected_grid(tmp_path):
    """Near the equator (cos(lat) = 1 to 1e-8) a geographic grid is the projected
    grid of spacing dx * 111111.1 m, up to the rounding of the spacings."""
    from oracle.oracle import Oracle

    def run(geo):
        sub = tmp_path / ("geo" if geo else "prj")
        sub.mkdir()
        m = synth.plain_regular(nmax=14, mmax=18, dx=300.0, tstop=1800.0, seed=4, nbumps=3)
        m.params.update(advection=1, coriolis=0)
        if geo:
            geographic(m, lon0=0.0, lat0=1.0e-4)
        d = m.write(str(sub))
        o = Oracle(d, "fp64")
        o.update(-1000.0, 100)
        return o.get("zs"), o.scalars()["t"]

    zg, tg = run(True)
    zp, tp = run(False)
    assert abs(tg - tp) < 1e-3 * tp
    assert np.abs(zg - zp).max() < 2e-3
