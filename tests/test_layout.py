"""Host-side layout of the B200 core against the oracle's literal index arrays.

The core replaces the reference's explicit uv index arrays
(sfincs_domain.f90:727-1261) by a dense grid with implicit neighbours and
per-cell flag bits.  These CPU tests check, cell by cell, that the flags encode
exactly the reference's face activity (kcuv), advection mask (mask_adv),
regular-cell mask (kcs), initial state and boundary-face lists.
"""
import os

import numpy as np
import pytest

from sfincs_b200 import bmi as B
from sfincs_b200 import synth

F_ACT, F_KCS1, F_UACT, F_VACT, F_UADV, F_VADV = 1, 2, 4, 8, 16, 32
F_CDN, F_CUP, F_CLF, F_CRT = 64, 128, 256, 512


def _oracle(d, prec="fp64"):
    from oracle.oracle import Oracle

    return Oracle(d, prec)


def _masks():
    def plain(**p):
        m = synth.plain_regular(nmax=14, mmax=17, dx=300.0, tstop=600.0, nbumps=5)
        m.params.update(p)
        return m

    out = {}
    out["plain"] = plain()
    m = plain(advection=1)
    m.msk[5:8, 6:9] = 0            # hole
    m.msk[0, 3:7] = 6              # lateral Neumann edge
    m.msk[-1, 9:12] = 3            # outflow cells
    m.msk[4, 0] = 0                # gap in the water-level boundary
    out["holes_neumann_outflow_adv"] = m
    m = plain(advection=1, advection_mask=0, theta=0.9)
    m.msk[2:4, 2:4] = 0
    out["adv_nomask_theta"] = m
    m = plain()
    m.bnd = np.array([[0.0, 500.0], [0.0, 3500.0], [0.0, 2000.0]])
    tb = m.bzs[:, 0]
    m.bzs = np.stack([tb, np.sin(tb / 3000.0), 0.5 * np.cos(tb / 2000.0), 0.2 + 0 * tb], axis=1)
    out["three_bnd_points"] = m
    m = plain(advection=1, theta=0.9)
    # a straight dam between columns 8 and 9 across the whole grid, a diagonal
    # one, and one along cell centres (touching points do not cut a face)
    m.thd = [np.array([[2400.0, -100.0], [2400.0, 14 * 300.0 + 100.0]]),
             np.array([[500.0, 500.0], [1700.0, 3100.0], [4100.0, 3500.0]]),
             np.array([[150.0, 1650.0], [1350.0, 1650.0]])]
    out["thin_dams"] = m
    return out


MASKS = _masks()


@pytest.mark.parametrize("name", sorted(MASKS))
def test_flags_match_oracle_index_arrays(tmp_path, name):
    d = MASKS[name].write(str(tmp_path))
    o = _oracle(d)
    s = o.scalars()
    n = int(s["np"])
    cnt = B.layout(d, "counts", 10)
    assert int(cnt[0]) == n and int(cnt[1]) == int(s["npuv"])
    assert cnt[6] == pytest.approx(s["dtmax"], rel=0, abs=0)
    assert cnt[7] == pytest.approx(s["dtmin"], rel=0, abs=0)
    assert cnt[8] == s["t0"] and cnt[9] == s["t1"]
    flags = B.layout(d, "flags", n).astype(np.int64)
    assert np.all(flags & F_ACT)
    assert np.array_equal((flags & F_KCS1) > 0, o.get("kcs") == 1)
    kcuv = o.get("kcuv")
    cell = o.get("uv_nm").astype(np.int64) - 1
    dirn = o.get("uv_dir").astype(np.int64)
    act = np.isin(kcuv, (1, 6))
    bit = np.where(dirn == 0, F_UACT, F_VACT)
    assert np.array_equal((flags[cell] & bit) > 0, act)
    if MASKS[name].params.get("advection", 0):
        madv = o.get("mask_adv")
        abit = np.where(dirn == 0, F_UADV, F_VADV)
        assert np.array_equal((flags[cell] & abit) > 0, madv == 1)
    # faces that do not exist in the reference are never active in the layout
    nfaces = ((flags & F_UACT) > 0).sum() + ((flags & F_VACT) > 0).sum()
    assert nfaces == act.sum()


@pytest.mark.parametrize("name", sorted(MASKS))
def test_boundary_faces_and_initial_state(tmp_path, name):
    d = MASKS[name].write(str(tmp_path))
    o = _oracle(d, "f32")
    s = o.scalars()
    cnt = B.layout(d, "counts", 10)
    nkb = int(cnt[3])
    kb_cell = B.layout(d, "kb_cell", nkb)
    kb_dir = B.layout(d, "kb_dir", nkb)
    kb_sign = B.layout(d, "kb_sign", nkb)
    assert np.array_equal(kb_cell, o.get("kb_cell", nkb))
    assert np.array_equal(kb_dir, o.get("kb_dir", nkb))
    assert np.array_equal(kb_sign, o.get("kb_sign", nkb))
    assert int(cnt[2]) == int(s["ngbnd"])
    zs = B.layout(d, "zs", int(s["np"]))
    assert np.array_equal(zs, o.get("zs"))


def test_subgrid_tables_and_volumes(tmp_path):
    m = synth.subgrid_regular(nmax=12, mmax=16, dx=400.0, P=6, tstop=1800.0, coast_x=2000.0)
    d = m.write(str(tmp_path))
    o = _oracle(d, "f32")
    n = int(o.scalars()["np"])
    cnt = B.layout(d, "counts", 10)
    assert int(cnt[4]) == 10
    assert np.array_equal(B.layout(d, "zs", n), o.get("zs"))
    assert np.array_equal(B.layout(d, "zvol", n), o.get("z_volume"))


def test_unsupported_inputs_are_refused(tmp_path):
    m = synth.plain_regular(nmax=6, mmax=7, dx=300.0, tstop=600.0, nbumps=1)
    m.params["netspwfile"] = "sfincs_spw.nc"
    d = m.write(str(tmp_path))
    with pytest.raises(RuntimeError, match="netspwfile"):
        B.layout(d, "counts", 10)


def test_thin_dam_faces(tmp_path):
    """The straight dam between columns 8 and 9 removes exactly the u faces of
    column 8 (both sides active) and leaves every v face; the oracle's kcuv
    agrees face by face with the layout (test_flags_match_oracle_index_arrays)."""
    m = synth.plain_regular(nmax=14, mmax=17, dx=300.0, tstop=600.0, nbumps=5)
    kcuv0 = _oracle(m.write(str(tmp_path / "open"))).get("kcuv")
    m.thd = [np.array([[2400.0, -100.0], [2400.0, 14 * 300.0 + 100.0]])]
    o = _oracle(m.write(str(tmp_path / "dam")))
    kcuv = o.get("kcuv")
    cell = o.get("uv_nm").astype(np.int64) - 1
    dirn = o.get("uv_dir").astype(np.int64)
    mcol = (np.flatnonzero(m.msk.ravel(order="F") > 0) // m.nmax + 1)[cell]  # 1-based column of each face's cell
    dammed = (kcuv == 0) & (kcuv0 != 0)
    assert np.array_equal(dammed & (dirn == 0), (dirn == 0) & (mcol == 8))
    assert not np.any(dammed & (dirn == 1))


def _weir_model():
    m = synth.plain_regular(nmax=14, mmax=17, dx=300.0, tstop=600.0, nbumps=5)
    m.params.update(advection=1, theta=0.9)
    m.weir = [np.array([[3000.0, -100.0, 2.0, 1.0], [3000.0, 2000.0, 3.0, 0.8], [3300.0, 4300.0, 1.0, 0.9]]),
              np.array([[700.0, 800.0, -20.0, 1.1], [2100.0, 3100.0, 5.0, 0.7]]),
              np.array([[300.0, 1000.0, 4.0, 1.0], [300.0, 2500.0, 4.0, 1.0]])]  # over the boundary column
    m.thd = [np.array([[2950.0, 500.0], [3050.0, 500.0]])]  # a dam under the weir: the weir wins
    return m


def test_weir_faces_match_oracle(tmp_path):
    """Weir faces (sfincs_structures.f90:38-381): which faces, their crest
    level, discharge coefficient and relative length, and the face activity
    (kcuv = 3 is not a momentum face) agree with the oracle bit for bit."""
    d = _weir_model().write(str(tmp_path))
    o = _oracle(d, "f32")
    n = int(o.get("nrstructures", 1)[0])
    assert n > 10
    assert int(B.layout(d, "nstruc", 1)[0]) == n
    so = o.get("struc", 4 * n).reshape(n, 4)
    sh = B.layout(d, "struc", 5 * n).reshape(n, 5)
    uv_nm = o.get("uv_nm").astype(np.int64) - 1
    uv_dir = o.get("uv_dir").astype(np.int64)
    ip = so[:, 0].astype(np.int64) - 1
    assert np.array_equal(uv_nm[ip], sh[:, 0].astype(np.int64))
    assert np.array_equal(uv_dir[ip], sh[:, 1].astype(np.int64))
    for k in range(3):
        assert np.array_equal(so[:, 1 + k].astype(np.float32), sh[:, 2 + k].astype(np.float32)), k
    flags = B.layout(d, "flags", int(o.scalars()["np"])).astype(np.int64)
    kcuv = o.get("kcuv")
    bit = np.where(uv_dir == 0, F_UACT, F_VACT)
    assert np.array_equal((flags[uv_nm] & bit) > 0, np.isin(kcuv, (1, 6)))
    assert np.count_nonzero(kcuv == 3) == n


@pytest.mark.parametrize("sub", [False, True], ids=["plain", "subgrid"])
def test_inifile_sets_initial_levels(tmp_path, sub):
    """A binary inifile (real*4 levels in cell order) sets zs = max(bed, ini)
    as set_initial_conditions does; levels below the bed are raised to it."""
    if sub:
        m = synth.subgrid_regular(nmax=12, mmax=14, dx=500.0, P=4, seed=5, tstop=600.0, coast_x=2000.0)
    else:
        m = synth.plain_regular(nmax=12, mmax=14, dx=300.0, tstop=600.0, nbumps=2)
    rng = np.random.default_rng(3)
    m.zsini_field = rng.uniform(-4.0, 3.0, size=m.msk.shape).astype(np.float32)
    d = m.write(str(tmp_path))
    o = _oracle(d, "f32")
    n = int(o.scalars()["np"])
    zs = B.layout(d, "zs", n)
    assert np.array_equal(zs, o.get("zs"))
    ini = m.compact(m.zsini_field).astype(np.float64)
    assert np.any(zs == ini) and np.any(zs > ini)  # some cells take the file's level, some the bed


def test_netcdf_inifile_is_refused(tmp_path):
    m = synth.plain_regular(nmax=6, mmax=7, dx=300.0, tstop=600.0, nbumps=1)
    m.params["inifile"] = "sfincs_ini.nc"
    d = m.write(str(tmp_path))
    with pytest.raises(RuntimeError, match="inifile"):
        B.layout(d, "counts", 10)


@pytest.mark.parametrize("sub", [False, True], ids=["plain", "subgrid"])
def test_downstream_river_faces_match_oracle(tmp_path, sub):
    """msk 5 cells become boundary faces in the reference's order (the east
    column here), and the model starts like the oracle."""
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_gpu_physics import _river

    d = _river(tmp_path, sub)
    o = _oracle(d, "f32")
    s = o.scalars()
    nb = int(s["nkcuv2"])
    n = int(s["np"])
    cnt = B.layout(d, "counts", 10)
    assert nb > 0
    kb = B.layout(d, "kb_cell", nb)
    assert np.array_equal(kb, o.get("kb_cell", nb))
    assert np.array_equal(B.layout(d, "zs", n), o.get("zs"))
    o.update(-1000.0, 20)
    assert np.isfinite(o.get("zs")).all()


def test_spiderweb_options_outside_the_core_are_refused(tmp_path):
    """Spiderweb reprojection (utmzone) and wind reduction over land (z0lfile)
    need tables and projections this core does not carry: refused at load."""
    from meteo_cases import add_spiderweb
    from sfincs_b200 import bmi as B

    for extra in ({"utmzone": "17N"}, {"z0lfile": "sfincs.z0l"}):
        d = tmp_path / list(extra)[0]
        d.mkdir()
        m = synth.plain_regular(nmax=10, mmax=12, dx=300.0, tstop=600.0, seed=1, nbumps=2)
        m.write(str(d))
        add_spiderweb(str(d), 3600.0, 3000.0, extra=extra)
        with pytest.raises(RuntimeError, match=list(extra)[0]):
            B.layout(str(d), "flags", 1)


def test_geographic_grids_load_and_refuse_what_they_do_not_carry(tmp_path):
    """crsgeo = 1 loads on regular grids; spiderwebs, weirs and drainage on a
    geographic grid are refused, naming the keyword."""
    from geo_cases import geographic

    m = synth.plain_regular(nmax=8, mmax=10, dx=300.0, tstop=600.0, seed=1, nbumps=2)
    geographic(m)
    d = m.write(str(tmp_path / "ok"))
    cnt = B.layout(d, "counts", 10)
    assert int(cnt[0]) == 80
    assert cnt[6] == 60.0 and cnt[7] == 0.0  # dtmax not limited by the spacing, no dtmin (sfincs_domain.f90:1403-1475)
    for key in ("spwfile", "weirfile", "drnfile"):
        m2 = synth.plain_regular(nmax=8, mmax=10, dx=300.0, tstop=600.0, seed=1, nbumps=2)
        geographic(m2)
        m2.params[key] = "x.dat"
        d2 = m2.write(str(tmp_path / key))
        with pytest.raises(RuntimeError, match=key):
            B.layout(d2, "counts", 10)
