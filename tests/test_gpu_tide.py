"""GPU parity of astronomic water-level boundaries (bca constituents added to
the boundary-point levels each step, sfincs_boundaries.f90:736-744) on
regular, subgrid and quadtree meshes, against the oracle in the core's
precision: the boundary cells' levels bit for bit, the rest within the usual
bar."""
import numpy as np
import pytest

from conftest import oracle_faces_to_cells
from tide_cases import add_bca, set_tref

pytestmark = pytest.mark.gpu

SETS_A0 = [[("A0", 0.12, 0.0), ("M2", 0.9, 35.0), ("S2", 0.3, 80.0), ("N2", 0.2, 10.0), ("K1", 0.15, 200.0),
            ("O1", 0.1, 150.0), ("M4", 0.05, 300.0)],
           [("A0", 0.08, 0.0), ("M2", 0.7, 50.0), ("S2", 0.25, 95.0), ("N2", 0.15, 20.0), ("K1", 0.12, 210.0),
            ("O1", 0.08, 160.0), ("M4", 0.04, 310.0)]]


def _model(d, variant=None):
    import os

    from sfincs_b200.bmi import Model

    old = os.environ.get("SFG_MOMENTUM_VARIANT")
    if variant is not None:
        os.environ["SFG_MOMENTUM_VARIANT"] = str(variant)
    try:
        return Model(d)
    finally:
        if variant is not None:
            if old is None:
                del os.environ["SFG_MOMENTUM_VARIANT"]
            else:
                os.environ["SFG_MOMENTUM_VARIANT"] = old


def _stepwise(d, variant, cells=None):
    from oracle.oracle import Oracle
    from sfincs_b200 import bmi as B

    o = Oracle(d, "f32")
    g = _model(d, variant)
    ngb = int(B.layout(d, "counts", 10)[2])
    gb = B.layout(d, "gb_cell", ngb).astype(np.int64)
    assert ngb > 0
    done = 0
    for n in (1, 1, 2, 6, 30, 60, 100):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        so, sg = o.scalars(), g.scalars()
        zs_o = o.get("zs") if cells is None else o.get("zs", cells[0])
        zs_g = g.get("zs")
        dzs = float(np.abs(zs_o - zs_g).max())
        if cells is None:
            qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
        else:
            q = o.get("q", cells[1])
            qx_o, qy_o = q[cells[2]], q[cells[3]]
        dq = max(float(np.abs(qx_o - g.get("qx")).max()), float(np.abs(qy_o - g.get("qy")).max()))
        print(f"v{variant} step {done}: t {so['t']:.3f}/{sg['t']:.3f} max|dzs| {dzs:.3g} max|dq| {dq:.3g}")
        assert sg["nt"] == so["nt"]
        assert abs(sg["t"] - so["t"]) <= 1e-6 * max(1.0, abs(so["t"]))
        assert np.array_equal(zs_g[gb], zs_o[gb].astype(np.float32)), done  # boundary levels bit for bit
        assert dzs <= 2e-5 and dq <= 2e-5, (done, dzs, dq)
    g.close()
    return o


@pytest.mark.parametrize("variant", [2, 5])
def test_two_points_with_bzs_and_a0_match_f32_oracle(tmp_path, variant):
    from sfincs_b200 import synth

    m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
    m.bnd = np.array([[0.0, 1200.0], [0.0, 8400.0]])
    m.bzs = np.stack([m.bzs[:, 0], 0.3 * m.bzs[:, 1], 0.2 * m.bzs[:, 1]], axis=1)
    m.params.update(advection=1)
    d = m.write(str(tmp_path))
    set_tref(d, "20210315 061530")
    add_bca(d, SETS_A0)
    _stepwise(d, variant)


def test_subgrid_without_bzs_matches_f32_oracle(tmp_path):
    from sfincs_b200 import synth

    m = synth.subgrid_regular(nmax=20, mmax=24, dx=500.0, P=8, seed=5, tstop=3600.0, rain_mmh=0.0,
                              rain_hours=0.5, coast_x=24 * 500.0 * 0.3, t_peak=1800.0, width_h=0.5,
                              surge_peak=1.5)
    m.bzs = None  # levels from the constituents alone
    m.prcp = None
    d = m.write(str(tmp_path))
    set_tref(d, "20180704 000000")
    add_bca(d, [[("M2", 1.1, 120.0), ("S2", 0.4, 140.0), ("K1", 0.2, 30.0), ("MF", 0.05, 0.0)]])
    _stepwise(d, 5)


def test_quadtree_matches_f32_oracle(tmp_path):
    from oracle.oracle import Oracle
    from sfincs_b200 import bmi as B
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=3600.0, subgrid=True, wind_speed=0.0, tide_period=1800.0)
    m.wnd = None
    d = m.write(str(tmp_path))
    set_tref(d, "20240101 000000")
    add_bca(d, [[("M2", 0.6, 45.0), ("K1", 0.2, 90.0), ("O1", 0.15, 60.0)]])
    qc = B.layout(d, "qt_counts", 4)
    npc, npq = int(qc[0]), int(qc[1]) + int(qc[2]) + 1
    o = Oracle(d, "f32")
    zmu = o.get("z_uv_mu", npc).astype(np.int64) - 1
    znu = o.get("z_uv_nu", npc).astype(np.int64) - 1
    o.close()
    _stepwise(d, None, cells=(npc, npq, zmu, znu))


def test_members_with_constituents_alone_equal_in_mix(tmp_path):
    """Two members with different constituents, dates and grids advanced by
    the same launches end bitwise where each ends alone."""
    from sfincs_b200 import synth
    from sfincs_b200.bmi import Ensemble, Model

    dirs = []
    for k, (tref, sets) in enumerate([("20210315 061530", SETS_A0),
                                      ("20180704 000000", [[("M2", 0.8, 10.0), ("K1", 0.2, 40.0)]])]):
        m = synth.plain_regular(nmax=20 + 4 * k, mmax=24 + 6 * k, dx=400.0, tstop=1800.0 + 600.0 * k, seed=3 + k,
                                nbumps=4)
        if len(sets) == 2:
            m.bnd = np.array([[0.0, 1200.0], [0.0, 6000.0]])
            m.bzs = np.stack([m.bzs[:, 0], 0.3 * m.bzs[:, 1], 0.2 * m.bzs[:, 1]], axis=1)
        d = m.write(str(tmp_path / f"m{k}"))
        set_tref(d, tref)
        add_bca(d, sets)
        dirs.append(d)
    e = Ensemble(dirs)
    e.run([e.scalars(i)["t1"] for i in range(len(dirs))])
    for i, d in enumerate(dirs):
        g = Model(d)
        g.run(g.scalars()["t1"])
        assert e.scalars(i)["nt"] == g.scalars()["nt"]
        for name in ("zs", "qx", "qy"):
            assert np.array_equal(e.get(i, name), g.get(name)), (i, name)
        g.close()
    e.close()
