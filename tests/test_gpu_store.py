"""GPU parity of the store variables (compute_store_variables,
sfincs_continuity.f90:626-720, and the time of the maximum level, :239-255):
maximum cell velocity and flux, wet duration and t_zsmax, on regular, subgrid
and quadtree meshes, against the oracle in the core's precision."""
import numpy as np
import pytest

from conftest import small_plain, small_subgrid

pytestmark = pytest.mark.gpu

STORE = dict(storevelmax=1, storefluxmax=1, storetwet=1, storetzsmax=1, twet_threshold=0.05)


def _compare(d, npc, steps=120):
    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model

    o = Oracle(d, "f32")
    g = Model(d)
    o.update(-1000.0, steps)
    g.step(steps)
    assert g.scalars()["nt"] == o.scalars()["nt"] == steps
    for name in ("zsmax", "vmax", "qmax", "twet", "tzsmax"):
        a, b = g.get(name).astype(np.float64), o.get(name, npc)
        print(f"{name}: range {b.min():.4g}..{b.max():.4g}, max|diff| {np.abs(a - b).max():.3g}")
        assert np.array_equal(a, b), name
    assert np.any(o.get("vmax", npc) > 0.0) and np.any(o.get("twet", npc) > 0.0)
    g.close()


@pytest.mark.parametrize("make", [small_plain, small_subgrid], ids=["plain", "subgrid"])
def test_store_variables_match_oracle(tmp_path, make):
    d, _ = make(tmp_path, advection=1, tstop=7200.0, **STORE)  # 120 steps end before tstop
    from oracle.oracle import Oracle

    _compare(d, int(Oracle(d, "f32").scalars()["np"]))


@pytest.mark.parametrize("subgrid", [False, True])
def test_quadtree_store_variables_match_oracle(tmp_path, subgrid):
    from sfincs_b200 import bmi as B
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=1800.0, subgrid=subgrid, wind_speed=30.0, tide_period=1800.0)
    m.params.update(STORE)
    d = m.write(str(tmp_path))
    _compare(d, int(B.layout(d, "qt_counts", 4)[0]))


@pytest.mark.parametrize("kind", ["cna", "cnb", "gai", "hor"])
def test_cumulative_rain_and_infiltration_match_oracle(tmp_path, kind):
    """Cumulative rain and infiltration (m) of every cell with each
    infiltration model with state (storecumprcp on)."""
    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model
    from test_gpu_physics import _infiltration_fields, _plain, _subgrid

    m = (_subgrid if kind in ("cnb", "hor") else _plain)(tmp_path, storecumprcp=1)
    d = _infiltration_fields(m, kind).write(str(tmp_path / kind))
    o = Oracle(d, "f32")
    g = Model(d)
    n = int(o.scalars()["np"])
    for steps in (30, 90):
        o.update(-1000.0, steps)
        g.step(steps)
        for name in ("zs", "cumprcp", "cuminf"):
            a, b = g.get(name).astype(np.float64), o.get(name, n)
            print(f"{kind} {name}: max {b.max():.4g} max|diff| {np.abs(a - b).max():.3g}")
            assert np.array_equal(a, b), name
    assert o.get("cuminf", n).max() > 0.0
    g.close()
