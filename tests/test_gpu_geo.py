"""GPU parity on geographic grids (crsgeo = 1): per-cell widths, areas and
Coriolis parameter on the per-thread kernels, stepwise against the oracle in
the core's precision, on plain and subgrid models with a boundary, advection,
Coriolis and rain."""
import numpy as np
import pytest

from conftest import oracle_faces_to_cells, small_plain, small_subgrid
from geo_cases import geographic

pytestmark = pytest.mark.gpu


def _write(tmp_path, subgrid):
    from sfincs_b200 import synth

    if subgrid:
        m = synth.subgrid_regular(nmax=20, mmax=24, dx=500.0, P=8, seed=5, tstop=3600.0, rain_mmh=40.0,
                                  rain_hours=0.5, coast_x=24 * 500.0 * 0.3, t_peak=1800.0, width_h=0.5,
                                  surge_peak=1.5)
    else:
        m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
        m.prcp = np.array([[0.0, 20.0], [3600.0, 20.0]])
    m.params.update(advection=1, coriolis=1, viscosity=1)
    geographic(m, lon0=-70.0, lat0=41.0)
    return m.write(str(tmp_path)), m


@pytest.mark.parametrize("subgrid", [False, True])
def test_geographic_matches_f32_oracle(tmp_path, subgrid):
    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model

    d, m = _write(tmp_path, subgrid)
    o = Oracle(d, "f32")
    g = Model(d)
    assert g.variant == 2  # geographic grids run the per-thread kernels
    done = 0
    for n in (1, 1, 2, 6, 30, 60, 100):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        so, sg = o.scalars(), g.scalars()
        dzs = float(np.abs(o.get("zs") - g.get("zs")).max())
        qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
        dq = max(float(np.abs(qx_o - g.get("qx")).max()), float(np.abs(qy_o - g.get("qy")).max()))
        print(f"geo sg={subgrid} step {done}: t {so['t']:.3f}/{sg['t']:.3f} max|dzs| {dzs:.3g} max|dq| {dq:.3g}")
        assert sg["nt"] == so["nt"]
        assert abs(sg["t"] - so["t"]) <= 1e-6 * max(1.0, abs(so["t"]))
        assert dzs <= 2e-5 and dq <= 2e-5, (done, dzs, dq)
    assert np.abs(qx_o).max() > 1e-3
    g.close()


def test_geographic_cell_area_through_the_bmi(tmp_path):
    """get_sfincs_cell_area gives cell_area_m2 on geographic grids (sfincs_bmi.f90:359-362)."""
    from oracle.oracle import Oracle
    from sfincs_b200.bmi import BMI

    d, m = _write(tmp_path, False)
    n = int(Oracle(d, "f32").scalars()["np"])
    area = Oracle(d, "f32").get("cell_area_m2", n)
    b = BMI()
    b.initialize(d)
    try:
        for k in (1, n // 2, n):
            assert b.get_sfincs_cell_area(k) == pytest.approx(float(area[k - 1]), rel=1e-7)
    finally:
        b.finalize()
