"""Pins of the CPU oracle (the checker).

The reference ships no tests or golden vectors and cannot be compiled here, so
the oracle is pinned by (1) an independent pure-Python restatement of the plain
step (tests/golden/pyref.py), (2) committed golden fixtures that freeze its
output on small seeded cases, and (3) analytic invariants of the scheme.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from sfincs_b200 import synth  # noqa: E402


def _oracle(d, prec="fp64"):
    from oracle.oracle import Oracle

    return Oracle(d, prec)


def test_oracle_matches_pure_python_restatement(tmp_path):
    from pyref import PyRef

    m = synth.plain_regular(nmax=6, mmax=8, dx=250.0, tstop=900.0, seed=11, nbumps=3)
    m.msk[3, 4] = 0
    d = m.write(str(tmp_path))
    o = _oracle(d, "fp64")
    bzs = np.loadtxt(os.path.join(d, "sfincs.bzs"))  # the values as written to the model file
    f = np.float32
    r = PyRef(m.msk, m.zb.astype(np.float64), 250.0, 250.0, zini=0.0, huthresh=0.01, alpha=0.5,
              gn2_sea=float(f(9.81) * (f(0.02) * f(0.02))), gn2_land=float(f(9.81) * (f(0.04) * f(0.04))),
              rgh_lev=0.0, t_bnd=bzs[:, 0].astype(np.float32).astype(np.float64),
              zs_bnd=bzs[:, 1].astype(np.float32).astype(np.float64))
    n_ = o.get("nm_n").astype(int) - 1
    m_ = o.get("nm_m").astype(int) - 1
    cell = o.get("uv_nm").astype(int) - 1
    dirn = o.get("uv_dir").astype(int)
    for step in range(40):
        o.update(-1.0)
        r.step()
        zs_r = np.array([r.zs[a][b] for a, b in zip(n_, m_)])
        q_r = np.array([(r.qu if d_ == 0 else r.qv)[(n_[c], m_[c])] for c, d_ in zip(cell, dirn)])
        s = o.scalars()
        assert s["t"] == pytest.approx(r.t, rel=1e-12)
        np.testing.assert_allclose(o.get("zs"), zs_r, rtol=0, atol=1e-9, err_msg=f"zs step {step}")
        np.testing.assert_allclose(o.get("q"), q_r, rtol=0, atol=1e-9, err_msg=f"q step {step}")


@pytest.mark.parametrize("name", ["plain_6x8", "subgrid_8x10"])
def test_golden_fixture(tmp_path, name):
    import make_golden

    case = {n: (m, k) for n, m, k in make_golden.cases()}[name]
    m, nsteps = case
    d = m.write(str(tmp_path))
    o = _oracle(d, "fp64")
    o.update(-1000.0, nsteps)
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    s = o.scalars()
    assert s["nt"] == g["nt"] and s["t"] == pytest.approx(float(g["t"]), rel=1e-13)
    np.testing.assert_allclose(o.get("zs"), g["zs"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(o.get("q"), g["q"], rtol=0, atol=1e-11)
    if "z_volume" in g:
        np.testing.assert_allclose(o.get("z_volume"), g["z_volume"], rtol=1e-12, atol=1e-8)


def _closed(m):
    m.msk[:, :] = np.where(m.msk > 0, 1, 0)
    m.bnd = None
    m.bzs = None
    return m


@pytest.mark.parametrize("prec", ["fp64", "ref", "f32"])
def test_lake_at_rest(tmp_path, prec):
    m = _closed(synth.plain_regular(nmax=10, mmax=12, dx=300.0, tstop=1200.0, nbumps=4))
    m.zb = np.minimum(m.zb, -1.0).astype(np.float32)
    m.params["zsini"] = 0.25
    d = m.write(str(tmp_path))
    o = _oracle(d, prec)
    z0 = o.get("zs")
    o.update(-1000.0, 100)
    assert np.array_equal(o.get("zs"), z0)
    assert np.all(o.get("q") == 0.0)


def test_dry_bed_stays_dry(tmp_path):
    m = _closed(synth.plain_regular(nmax=8, mmax=9, dx=300.0, tstop=1200.0, nbumps=2))
    m.zb = (m.zb + 20.0).astype(np.float32)  # everything above zsini
    d = m.write(str(tmp_path))
    o = _oracle(d)
    z0 = o.get("zs")
    o.update(-1000.0, 50)
    assert np.array_equal(o.get("zs"), z0)


def test_closed_basin_conserves_volume_regular(tmp_path):
    m = _closed(synth.plain_regular(nmax=12, mmax=14, dx=200.0, tstop=3600.0, nbumps=5))
    m.zb = np.minimum(m.zb, -0.5).astype(np.float32)
    m.params["advection"] = 1
    d = m.write(str(tmp_path))
    o = _oracle(d)
    zs = o.get("zs")
    zs = zs + 0.5 * np.exp(-np.arange(zs.size) / 40.0)  # a mound of water
    o.set("zs", zs)
    zb = o.get("zb")
    v0 = np.sum(o.get("zs") - zb)
    o.update(-1000.0, 300)
    v1 = np.sum(o.get("zs") - zb)
    assert abs(v1 - v0) <= 1e-10 * abs(v0)
    assert np.abs(o.get("q")).max() > 0  # water moved


def test_rain_on_flat_closed_basin(tmp_path):
    m = _closed(synth.plain_regular(nmax=6, mmax=7, dx=200.0, tstop=3600.0, nbumps=0))
    m.zb = np.full_like(m.zb, -2.0)
    m.prcp = np.array([[0.0, 36.0], [7200.0, 36.0]])  # 36 mm/h = 1e-5 m/s
    d = m.write(str(tmp_path))
    o = _oracle(d)
    o.update(-1000.0, 60)
    s = o.scalars()
    zs = o.get("zs")
    # every cell gained P * (t - t0); the rain rate is the real*4 value of 36 mm/h in m/s
    p = float(np.float32(36.0) / np.float32(1000 * 3600))
    assert np.ptp(zs) <= 1e-12
    # (the time interpolation of the rain series is done in real*4: ~1e-7 relative wobble)
    assert zs[0] - 0.0 == pytest.approx(p * (s["t"] - s["t0"]), rel=2e-7)


def test_symmetric_dam_break(tmp_path):
    m = _closed(synth.plain_regular(nmax=9, mmax=16, dx=100.0, tstop=3600.0, nbumps=0))
    m.zb = np.full_like(m.zb, -1.0)
    d = m.write(str(tmp_path))
    o = _oracle(d)
    n = o.get("nm_n").astype(int)
    mm = o.get("nm_m").astype(int)
    zs = np.where(mm <= 8, 1.0, 0.0)
    o.set("zs", zs)
    o.update(-1000.0, 80)
    z = o.get("zs")
    grid = np.zeros((9, 16))
    grid[n - 1, mm - 1] = z
    # mirror symmetry across the channel axis (n -> 10 - n)
    np.testing.assert_allclose(grid, grid[::-1, :], rtol=0, atol=1e-12)
    assert grid[:, 12].max() > 0.0  # the front travelled east


def test_thin_dam_holds_a_dam_break(tmp_path):
    """A thin dam across the channel (sfincs_structures.f90:385-495): the front
    of a dam break reaches it and nothing crosses; the water behind it keeps
    its volume."""
    m = _closed(synth.plain_regular(nmax=9, mmax=16, dx=100.0, tstop=3600.0, nbumps=0))
    m.zb = np.full_like(m.zb, -1.0)
    m.thd = [np.array([[1200.0, -50.0], [1200.0, 950.0]])]  # between columns 12 and 13
    d = m.write(str(tmp_path))
    o = _oracle(d)
    mm = o.get("nm_m").astype(int)
    o.set("zs", np.where(mm <= 6, 1.0, 0.0))
    v0 = np.sum(o.get("zs") + 1.0)
    o.update(-1000.0, 400)
    z = o.get("zs")
    assert np.all(z[mm >= 13] == 0.0)
    assert z[mm == 12].max() > 0.05  # the front arrived at the dam
    assert abs(np.sum(z + 1.0) - v0) <= 1e-10 * v0


def test_weir_free_and_submerged_flow(tmp_path):
    """Broad-crested weir (sfincs_structures.f90:592-697) in a closed basin:
    after one step the flux over every weir face is the free-flow discharge
    Cd 1.7049 h1^1.5, or the submerged one Cd h2 sqrt(2 g (h1 - h2)), times
    the crossed length, from the levels at the start of the step."""
    m = _closed(synth.plain_regular(nmax=8, mmax=12, dx=100.0, tstop=3600.0, nbumps=0))
    m.zb = np.full_like(m.zb, -2.0)
    m.weir = [np.array([[600.0, -50.0, 0.0, 0.9], [600.0, 850.0, 0.0, 0.9]])]  # between columns 6 and 7
    d = m.write(str(tmp_path))
    o = _oracle(d)
    assert int(o.get("nrstructures", 1)[0]) == 8
    mm = o.get("nm_m").astype(int)
    nn = o.get("nm_n").astype(int)
    # rows 1-4: free flow (east below the crest); rows 5-8: submerged
    zs = np.where(mm <= 6, 0.5, np.where(nn <= 4, -0.5, 0.45))
    o.set("zs", zs)
    o.update(-1000.0, 1)
    q = o.get("q")
    st = o.get("struc", 32).reshape(8, 4)
    nmu = o.get("uv_nmu").astype(int) - 1
    for ip, crest, cd, rel in st:
        ip = int(ip) - 1
        h1 = 0.5 - crest
        h2 = zs[nmu[ip]] - crest  # the east neighbour, column 7
        if h2 > 2.0 / 3.0 * h1:
            want = cd * h2 * np.sqrt(2.0 * 9.81 * (h1 - h2))
        else:
            want = cd * 1.7049 * h1 ** 1.5
        assert q[ip] == pytest.approx(want * rel, rel=1e-6)
        assert rel == pytest.approx(1.0, abs=1e-6)


def test_drainage_structures_move_water_and_conserve_volume(tmp_path):
    """Drainage structures (sfincs_discharges.f90:370-657) in a closed basin: a
    pump, a culvert, a check valve and two gates move water between cells;
    the FP64 volume is unchanged, and the pump's intake loses water while its
    outfall gains it."""
    m = _closed(synth.plain_regular(nmax=10, mmax=14, dx=100.0, tstop=3600.0, nbumps=0))
    m.zb = np.full_like(m.zb, -2.0)
    m.drn = [(250.0, 250.0, 1150.0, 850.0, 1, 0.5),        # pump 0.5 m3/s
             (550.0, 150.0, 550.0, 950.0, 2, 0.3),         # culvert
             (950.0, 150.0, 150.0, 950.0, 3, 0.4),         # check valve
             (1250.0, 350.0, 1250.0, 750.0, 4, 2.0, -1.0, 0.02, -0.5, 5.0, 60.0),   # level-controlled gate
             (750.0, 550.0, 350.0, 550.0, 5, 1.5, -1.5, 0.025, 300.0, 900.0, 30.0)]  # time-controlled gate
    d = m.write(str(tmp_path))
    o = _oracle(d)
    n = o.get("nm_n").astype(int)
    mm = o.get("nm_m").astype(int)
    zs = 0.1 * np.sin(n / 2.0) + 0.05 * np.cos(mm / 3.0)
    o.set("zs", zs)
    v0 = np.sum(o.get("zs") + 2.0)
    o.update(-1000.0, 300)
    z = o.get("zs")
    assert abs(np.sum(z + 2.0) - v0) <= 1e-9 * v0
    cell = lambda x, y: int(np.flatnonzero((n == int(y // 100) + 1) & (mm == int(x // 100) + 1))[0])
    assert z[cell(250.0, 250.0)] < zs[cell(250.0, 250.0)]
    assert z[cell(1150.0, 850.0)] > zs[cell(1150.0, 850.0)]


def test_h73table_follows_the_power(tmp_path):
    """hu**(7/3) from the lookup table (3 significant digits of hu) moves the
    plain case by a fraction of a millimetre against the exact power over 100
    steps, at every precision."""
    for prec in ("ref", "f32", "fp64"):
        d1 = str(tmp_path / f"a{prec}")
        d2 = str(tmp_path / f"b{prec}")
        for d, on in ((d1, 0), (d2, 1)):
            m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=1800.0, seed=3, nbumps=6)
            m.params["h73table"] = on
            m.write(d)
        a, b = _oracle(d1, prec), _oracle(d2, prec)
        a.update(-1000.0, 100)
        b.update(-1000.0, 100)
        dz = np.abs(a.get("zs") - b.get("zs")).max()
        assert 0.0 < dz <= 1e-3, (prec, dz)
