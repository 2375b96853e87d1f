"""GPU parity of the gridded meteo forcing (ASCII amu/amv wind, amp pressure,
ampr rain; update windows every dtwnd, per-step blending, spin-up, the
pressure-gradient term and the barometric boundary correction) on regular,
subgrid and quadtree meshes, against the oracle in the core's precision."""
import numpy as np
import pytest

from conftest import oracle_faces_to_cells
from meteo_cases import add_meteo

pytestmark = pytest.mark.gpu


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


def _regular(tmp_path, subgrid, **params):
    from sfincs_b200 import synth

    if subgrid:
        m = synth.subgrid_regular(nmax=20, mmax=24, dx=500.0, P=8, seed=5, tstop=3600.0, rain_mmh=40.0,
                                  rain_hours=0.5, coast_x=24 * 500.0 * 0.3, t_peak=1800.0, width_h=0.5,
                                  surge_peak=1.5)
        m.prcp = None  # rain comes from the grid
    else:
        m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
    m.params.update(advection=1, **params)
    d = m.write(str(tmp_path))
    add_meteo(d, m.mmax * m.dx, m.nmax * m.dy, extra={"spinup_meteo": 1} if params.get("tspinup") else None)
    return d


def _stepwise(d, variant, cells=None, t_min=1200.0):
    from oracle.oracle import Oracle

    o = Oracle(d, "f32")
    g = _model(d, variant)
    done = 0
    for n in (1, 1, 2, 6, 30, 60, 100):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        so, sg = o.scalars(), g.scalars()
        zs_o = o.get("zs") if cells is None else o.get("zs", cells[0])
        dzs = float(np.abs(zs_o - g.get("zs")).max())
        if cells is None:
            qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
        else:
            q = o.get("q", cells[1])
            qx_o, qy_o = q[cells[2]], q[cells[3]]
        dq = max(float(np.abs(qx_o - g.get("qx")).max()), float(np.abs(qy_o - g.get("qy")).max()))
        print(f"v{variant} step {done}: t {so['t']:.3f}/{sg['t']:.3f} max|dzs| {dzs:.3g} max|dq| {dq:.3g}")
        assert sg["nt"] == so["nt"]
        assert abs(sg["t"] - so["t"]) <= 1e-6 * max(1.0, abs(so["t"]))
        assert dzs <= 2e-5 and dq <= 2e-5, (done, dzs, dq)
    assert so["t"] > t_min  # at least two update windows passed
    g.close()


@pytest.mark.parametrize("variant", [2, 5])
@pytest.mark.parametrize("subgrid", [False, True])
def test_gridded_meteo_matches_f32_oracle(tmp_path, subgrid, variant):
    _stepwise(_regular(tmp_path, subgrid), variant)


def test_gridded_meteo_spinup_matches_f32_oracle(tmp_path):
    _stepwise(_regular(tmp_path, False, tspinup=900.0), 5)


@pytest.mark.parametrize("subgrid", [False, True])
def test_quadtree_gridded_meteo_matches_f32_oracle(tmp_path, subgrid):
    from oracle.oracle import Oracle
    from sfincs_b200 import bmi as B
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=3600.0, subgrid=subgrid, wind_speed=0.0, tide_period=1800.0)
    m.wnd = None
    d = m.write(str(tmp_path))
    add_meteo(d, 10 * 400.0, 8 * 400.0, dt_rec=300.0, dtwnd=150.0)  # the fine levels take short steps
    qc = B.layout(d, "qt_counts", 4)
    npc, npq = int(qc[0]), int(qc[1]) + int(qc[2]) + 1
    o = Oracle(d, "f32")
    zmu = o.get("z_uv_mu", npc).astype(np.int64) - 1
    znu = o.get("z_uv_nu", npc).astype(np.int64) - 1
    o.close()
    _stepwise(d, None, cells=(npc, npq, zmu, znu), t_min=300.0)


def _spw_regular(tmp_path, subgrid, background):
    from meteo_cases import add_spiderweb
    from sfincs_b200 import synth

    if subgrid:
        m = synth.subgrid_regular(nmax=20, mmax=24, dx=500.0, P=8, seed=5, tstop=3600.0, rain_mmh=40.0,
                                  rain_hours=0.5, coast_x=24 * 500.0 * 0.3, t_peak=1800.0, width_h=0.5,
                                  surge_peak=1.5)
        m.prcp = None  # rain comes from the web (and the grid)
    else:
        m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
    m.params.update(advection=1)
    d = m.write(str(tmp_path))
    if background:
        add_meteo(d, m.mmax * m.dx, m.nmax * m.dy)
    add_spiderweb(d, m.mmax * m.dx, m.nmax * m.dy, extra={"spwmergefrac": 0.6})
    return d


@pytest.mark.parametrize("variant", [2, 5])
def test_spiderweb_matches_f32_oracle(tmp_path, variant):
    """A cyclone's polar wind, pressure and rain alone (faded in and out)."""
    _stepwise(_spw_regular(tmp_path, False, False), variant)


def test_spiderweb_over_gridded_meteo_matches_f32_oracle(tmp_path):
    """A cyclone merged over amu/amv/amp/ampr background fields on a subgrid model."""
    _stepwise(_spw_regular(tmp_path, True, True), 5)


def test_quadtree_spiderweb_matches_f32_oracle(tmp_path):
    from meteo_cases import add_spiderweb
    from oracle.oracle import Oracle
    from sfincs_b200 import bmi as B
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=3600.0, subgrid=True, wind_speed=0.0, tide_period=1800.0)
    m.wnd = None
    d = m.write(str(tmp_path))
    add_spiderweb(d, 10 * 400.0, 8 * 400.0, t_first=100.0, dt_rec=150.0, dtwnd=100.0)
    qc = B.layout(d, "qt_counts", 4)
    npc, npq = int(qc[0]), int(qc[1]) + int(qc[2]) + 1
    o = Oracle(d, "f32")
    zmu = o.get("z_uv_mu", npc).astype(np.int64) - 1
    znu = o.get("z_uv_nu", npc).astype(np.int64) - 1
    o.close()
    _stepwise(d, None, cells=(npc, npq, zmu, znu), t_min=200.0)
