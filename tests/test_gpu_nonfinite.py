"""Non-finite state stays inside the tables.

A model that goes unstable fills its state with inf and NaN.  The reference
keeps stepping such a model until its dt falls below dtmin
(sfincs_lib.f90:634-648).  The GPU core must do the same without reading
outside any array.  The subgrid lookups are the only places where state
becomes an index.  A NaN volume fails both guards of the volume-to-level
inversion (sfincs_continuity.f90:556-569) and reaches int(v / dzvol) + 1.
These tests plant a NaN in one cell's external source term (qext), so the
cell's FP64 volume turns NaN on the next step.  Each continuity kernel (TMA
tiles, per-thread loads, quadtree) must then run on with no CUDA error.  The
NaN must spread only through the flux stencil.  A fresh model on the same
device must still match the oracle.
"""
import numpy as np
import pytest

from conftest import small_subgrid

pytestmark = pytest.mark.gpu


def _model(d, variant, bmi):
    import os

    from sfincs_b200.bmi import Model

    old = os.environ.get("SFG_MOMENTUM_VARIANT")
    if variant is not None:
        os.environ["SFG_MOMENTUM_VARIANT"] = str(variant)
    try:
        return Model(d, bmi=bmi)
    finally:
        if variant is not None:
            if old is None:
                del os.environ["SFG_MOMENTUM_VARIANT"]
            else:
                os.environ["SFG_MOMENTUM_VARIANT"] = old


def _plant_nan_and_step(g, cell, steps):
    n = int(g.scalars()["np"])
    qext = np.zeros(n, np.float32)
    qext[cell] = np.nan
    g.set("qext", qext)
    g.step(steps)
    g.sync()
    return g.get("zs"), g.get("z_volume")


@pytest.mark.parametrize("variant", [5, 2])
def test_nan_volume_regular_subgrid(tmp_path, variant):
    d, _ = small_subgrid(tmp_path, tstop=7200.0)
    g = _model(d, variant, bmi=True)
    g.step(20)
    zs0 = g.get("zs")
    wet = np.flatnonzero(np.isfinite(zs0) & (g.get("z_volume") > 1.0))
    assert wet.size, "the test model has no wet cell to plant the NaN in"
    cell = int(wet[wet.size // 2])
    zs, vol = _plant_nan_and_step(g, cell, 30)
    assert np.isnan(vol[cell]), "the planted NaN did not reach the cell's volume"
    assert np.isfinite(zs).sum() > 0
    s = g.scalars()
    assert s["nt"] >= 50
    g.close()


def test_nan_volume_quadtree_subgrid(tmp_path):
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=3600.0, subgrid=True, wind_speed=30.0, tide_period=1800.0)
    d = tmp_path / "qt"
    d.mkdir()
    d = m.write(str(d))
    g = _model(d, None, bmi=True)
    g.step(20)
    wet = np.flatnonzero(g.get("z_volume") > 1.0)
    assert wet.size
    cell = int(wet[wet.size // 2])
    zs, vol = _plant_nan_and_step(g, cell, 30)
    assert np.isnan(vol[cell])
    assert np.isfinite(zs).sum() > 0
    g.close()


def test_device_healthy_after_nan_models(tmp_path):
    """After the NaN models above, a fresh model on the same device still
    matches the oracle in the core's precision."""
    from oracle.oracle import Oracle

    d, _ = small_subgrid(tmp_path)
    g = _model(d, None, bmi=False)
    o = Oracle(d, "f32")
    o.update(-1000.0, 40)
    g.step(40)
    assert float(np.abs(o.get("zs") - g.get("zs")).max()) <= 2e-5
    g.close()
