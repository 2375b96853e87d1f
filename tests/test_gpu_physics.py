"""GPU parity of the optional physics, term by term.

The main parity tests (test_gpu_parity.py) run the default switches. Here each
case turns on terms that those leave off: Coriolis, wind stress from a time
series, theta smoothing, the "original" advection scheme, the slope limiter,
friction2d off, viscosity and no wiggle suppression on a subgrid model, c2d
infiltration and the infiltration models with state (curve number with and
without recovery, Green-Ampt, Horton), point sources, Neumann and outflow boundary cells, thin dams,
weirs, the five drainage structure types, the hu**(7/3) lookup table and
initial levels from an inifile (regular and subgrid). For each
case the CUDA core is compared with the oracle in the core's own precision
after 1, 2, 4, 10, 40 and 100 steps, on the default kernel path and on the
per-thread-load path. The bars are those of the main stepwise test: time
within 1e-6 relative, zs and q within 2e-5.  Every kernel path must also store
the same bits as every other on each case.
"""
import numpy as np
import pytest

from conftest import oracle_faces_to_cells

pytestmark = pytest.mark.gpu


def _plain(tmp_path, **params):
    from sfincs_b200 import synth

    m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
    m.params.update(params)
    return m


def _subgrid(tmp_path, **params):
    from sfincs_b200 import synth

    m = synth.subgrid_regular(nmax=20, mmax=24, dx=500.0, P=8, seed=5, tstop=3600.0, rain_mmh=40.0, rain_hours=0.5,
                              coast_x=24 * 500.0 * 0.3, t_peak=1800.0, width_h=0.5, surge_peak=1.5)
    m.params.update(params)
    return m


def _wind(tstop=3600.0):
    # t, speed (m/s), nautical direction (from)
    return np.array([[0.0, 12.0, 270.0], [900.0, 20.0, 240.0], [tstop + 600.0, 8.0, 300.0]])


def case_coriolis_wind_theta(tmp_path):
    m = _plain(tmp_path, advection=1, latitude=45.0, theta=0.9)
    m.wnd = _wind()
    return m


def case_original_advection_slopelim_nofric2d(tmp_path):
    return _plain(tmp_path, advection=1, advection_scheme="original", slopelim=0.05, friction2d=0)


def case_boundary_kinds(tmp_path):
    m = _plain(tmp_path, advection=1)
    m.msk[0, 5:12] = 6    # Neumann edge
    m.msk[-1, 8:14] = 3   # outflow cells
    return m


def case_plain_infiltration(tmp_path):
    m = _plain(tmp_path)
    rng = np.random.default_rng(7)
    m.qinf_field = rng.uniform(0.0, 20.0, size=m.msk.shape).astype(np.float32)  # mm/h
    m.prcp = np.array([[0.0, 30.0], [3600.0, 30.0]])
    return m


def case_subgrid_visc_nowiggle(tmp_path):
    return _subgrid(tmp_path, advection=1, viscosity=1, wiggle_suppression=0)


def case_subgrid_infiltration_sources(tmp_path):
    m = _subgrid(tmp_path, advection=1)
    rng = np.random.default_rng(11)
    m.qinf_field = rng.uniform(0.0, 10.0, size=m.msk.shape).astype(np.float32)
    # three point sources inside the domain (x, y in metres), discharges in m3/s
    m.src = np.array([[6000.0, 3000.0], [9000.0, 6000.0], [4500.0, 8000.0]])
    m.dis = np.array([[0.0, 5.0, 0.0, 2.0], [1800.0, 20.0, 3.0, 2.0], [4200.0, 0.0, 6.0, 2.0]])
    return m


def case_thin_dams_theta(tmp_path):
    m = _plain(tmp_path, advection=1, theta=0.9)
    # a dam across the domain between columns 15 and 16 with a gap, and a diagonal one
    m.thd = [np.array([[6000.0, -200.0], [6000.0, 5000.0]]),
             np.array([[2000.0, 2000.0], [4400.0, 7000.0], [9000.0, 8000.0]])]
    return m


def case_subgrid_thin_dams(tmp_path):
    m = _subgrid(tmp_path, advection=1)
    m.thd = [np.array([[5000.0, -100.0], [5000.0, 6500.0], [7000.0, 9000.0]])]
    return m


def case_weirs(tmp_path):
    m = _plain(tmp_path, advection=1, theta=0.9)
    # a weir across the channel with a varying crest, one over the boundary
    # column, and a thin dam under the first weir (the weir wins)
    m.weir = [np.array([[6000.0, -200.0, -1.0, 1.0], [6000.0, 5000.0, 0.5, 0.8], [7000.0, 9800.0, -2.0, 0.9]]),
              np.array([[400.0, 2000.0, 1.5, 1.0], [400.0, 6000.0, 1.5, 1.0]])]
    m.thd = [np.array([[5800.0, 3000.0], [6200.0, 3000.0]])]
    return m


def case_subgrid_weirs(tmp_path):
    m = _subgrid(tmp_path, advection=1)
    m.weir = [np.array([[5000.0, -100.0, 0.5, 1.0], [5000.0, 10100.0, 2.5, 1.0]])]
    return m


_DRAINAGE = [(1000.0, 1000.0, 3000.0, 3000.0, 1, 2.0),                  # pump
             (2200.0, 5000.0, 4200.0, 7000.0, 2, 1.5),                  # culvert
             (1400.0, 8200.0, 600.0, 4600.0, 3, 1.0),                   # check valve
             (3400.0, 1800.0, 1800.0, 3400.0, 4, 3.0, -6.0, 0.02, -3.0, 4.0, 120.0),   # level-controlled gate
             (2600.0, 2600.0, 600.0, 600.0, 5, 2.0, -8.0, 0.025, 900.0, 2400.0, 60.0)]  # time-controlled gate


def case_drainage(tmp_path):
    m = _plain(tmp_path)
    m.drn = _DRAINAGE
    return m


def case_subgrid_drainage(tmp_path):
    m = _subgrid(tmp_path, advection=1)
    m.drn = _DRAINAGE
    return m


def case_h73table(tmp_path):
    return _plain(tmp_path, advection=1, h73table=1)


def case_subgrid_h73table(tmp_path):
    return _subgrid(tmp_path, advection=1, h73table=1)


def _infiltration_fields(m, kind, seed=17):
    """Per-cell parameter files of an infiltration model with state."""
    rng = np.random.default_rng(seed)
    shp = m.msk.shape
    if kind == "cna":
        m.cell_fields["scsfile"] = rng.uniform(0.05, 2.0, shp)
    elif kind == "cnb":
        m.cell_fields["smaxfile"] = rng.uniform(0.005, 0.05, shp)
        m.cell_fields["sefffile"] = rng.uniform(0.002, 0.03, shp)
        m.cell_fields["ksfile"] = rng.uniform(10.0, 20000.0, shp)
    elif kind == "gai":
        m.cell_fields["psifile"] = rng.uniform(50.0, 300.0, shp)
        m.cell_fields["sigmafile"] = rng.uniform(0.1, 0.4, shp)
        m.cell_fields["ksfile"] = rng.uniform(5.0, 20000.0, shp)
    else:
        m.cell_fields["fcfile"] = rng.uniform(5.0, 20.0, shp)
        m.cell_fields["f0file"] = rng.uniform(50.0, 150.0, shp)
        m.cell_fields["kdfile"] = rng.uniform(1.0, 5.0, shp)
    # rain that stops early, so the recovery branches run too
    m.prcp = np.array([[0.0, 40.0], [400.0, 40.0], [401.0, 0.0], [7200.0, 0.0]])
    return m


def case_infiltration_cna(tmp_path):
    return _infiltration_fields(_plain(tmp_path, storecumprcp=1), "cna")


def case_subgrid_infiltration_cnb(tmp_path):
    return _infiltration_fields(_subgrid(tmp_path, advection=1), "cnb")


def case_infiltration_gai(tmp_path):
    return _infiltration_fields(_plain(tmp_path, advection=1), "gai")


def case_subgrid_infiltration_gai(tmp_path):
    return _infiltration_fields(_subgrid(tmp_path), "gai")


def case_infiltration_hor(tmp_path):
    return _infiltration_fields(_plain(tmp_path), "hor")


def case_subgrid_infiltration_hor(tmp_path):
    return _infiltration_fields(_subgrid(tmp_path, storecumprcp=1), "hor")


def case_inifile(tmp_path):
    m = _plain(tmp_path, advection=1)
    ini = np.full(m.msk.shape, -1.0, np.float32)
    ini[:, : m.mmax // 2] = 1.5  # initial levels from a file: a dam break across the middle
    m.zsini_field = ini
    return m


def case_subgrid_inifile(tmp_path):
    m = _subgrid(tmp_path, advection=1)
    m.zsini_field = np.where(np.arange(m.mmax)[None, :] < m.mmax // 3, 2.0, 0.0).repeat(m.nmax, 0).astype(np.float32)
    return m


CASES = {f.__name__[5:]: f for f in (case_infiltration_cna, case_subgrid_infiltration_cnb, case_infiltration_gai,
                                      case_subgrid_infiltration_gai, case_infiltration_hor,
                                      case_subgrid_infiltration_hor, case_inifile, case_subgrid_inifile, case_h73table, case_subgrid_h73table, case_coriolis_wind_theta, case_original_advection_slopelim_nofric2d,
                                      case_boundary_kinds, case_plain_infiltration, case_subgrid_visc_nowiggle,
                                      case_subgrid_infiltration_sources, case_thin_dams_theta,
                                      case_subgrid_thin_dams, case_weirs, case_subgrid_weirs, case_drainage,
                                      case_subgrid_drainage)}


def _model(d, variant):
    import os

    from sfincs_b200.bmi import Model

    old = os.environ.get("SFG_MOMENTUM_VARIANT")
    os.environ["SFG_MOMENTUM_VARIANT"] = str(variant)
    try:
        return Model(d)
    finally:
        if old is None:
            del os.environ["SFG_MOMENTUM_VARIANT"]
        else:
            os.environ["SFG_MOMENTUM_VARIANT"] = old


@pytest.mark.parametrize("variant", [2, 5])
@pytest.mark.parametrize("kind", sorted(CASES))
def test_physics_stepwise_matches_f32_oracle(tmp_path, kind, variant):
    from oracle.oracle import Oracle

    d = CASES[kind](tmp_path).write(str(tmp_path / kind))
    o = Oracle(d, "f32")
    g = _model(d, variant)
    done = 0
    for n in (1, 1, 2, 6, 30, 60):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        so, sg = o.scalars(), g.scalars()
        dzs = float(np.abs(o.get("zs") - g.get("zs")).max())
        qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
        dq = max(float(np.abs(qx_o - g.get("qx")).max()), float(np.abs(qy_o - g.get("qy")).max()))
        print(f"{kind} v{variant} step {done}: dt {so['dt']:.6g}/{sg['dt']:.6g} max|dzs| {dzs:.3g} max|dq| {dq:.3g}")
        assert sg["nt"] == so["nt"]
        assert abs(sg["t"] - so["t"]) <= 1e-6 * max(1.0, abs(so["t"]))
        assert dzs <= 2e-5, f"{kind}: zs differs by {dzs} after {done} steps"
        assert dq <= 2e-5, f"{kind}: q differs by {dq} after {done} steps"
    g.close()


@pytest.mark.parametrize("kind", sorted(CASES))
def test_physics_paths_agree_bitwise(tmp_path, kind):
    """The TMA-staged tile kernels (5, 4) and the per-thread kernel (2) store
    the same bits with every optional term switched on."""
    d = CASES[kind](tmp_path).write(str(tmp_path / kind))
    runs = [_model(d, v) for v in (5, 4, 2)]
    for g in runs:
        g.step(100)
    for name in ("zs", "qx", "qy", "uvx", "uvy"):
        for v, g in zip((4, 2), runs[1:]):
            assert np.array_equal(runs[0].get(name), g.get(name)), f"{name}: variant {v} differs from 5"
    for g in runs:
        g.close()


def _river(tmp_path, subgrid=False):
    """A channel deepening to the east: tide on the west column, a downstream
    river boundary (msk 5) on the east column whose level follows the water
    two cells inside, lowered by the bed slope times the distance."""
    import os

    if subgrid:
        m = _subgrid(tmp_path, advection=1)
    else:
        m = _plain(tmp_path, advection=1)
        x = (np.arange(m.mmax) + 0.5) * m.dx
        m.zb = (np.full(m.msk.shape, -3.0) - 0.0002 * x[None, :]).astype(np.float32)
    m.msk[:, -1] = 5
    d = m.write(str(tmp_path / ("river_sg" if subgrid else "river")))
    xe = m.mmax * m.dx - 0.5 * m.dx
    rows = []
    for n in (2, m.nmax // 2, m.nmax - 3):
        y = (n + 0.5) * m.dx
        rows.append(f"{xe:.3f} {y:.3f} {xe - 2 * m.dx:.3f} {y:.3f} 0.0002 -1.0")
    rows.append(f"{xe:.3f} {m.nmax * m.dx * 0.9:.3f} {xe - 3 * m.dx:.3f} {m.nmax * m.dx * 0.9:.3f} 0.0001 1000.0")
    with open(os.path.join(d, "sfincs.bdr"), "w") as f:
        f.write("\n".join(rows) + "\n")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'bdrfile':<20} = sfincs.bdr\n")
    return d


@pytest.mark.parametrize("subgrid", [False, True])
@pytest.mark.parametrize("variant", [2, 5])
def test_downstream_river_boundary_matches_f32_oracle(tmp_path, subgrid, variant):
    """Downstream river boundary cells (kcs 5, sfincs_boundaries.f90:878-902)."""
    from oracle.oracle import Oracle

    d = _river(tmp_path, subgrid)
    o = Oracle(d, "f32")
    g = _model(d, variant)
    done = 0
    for n in (1, 1, 2, 6, 30, 60):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        dzs = float(np.abs(o.get("zs") - g.get("zs")).max())
        qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
        dq = max(float(np.abs(qx_o - g.get("qx")).max()), float(np.abs(qy_o - g.get("qy")).max()))
        print(f"river subgrid={subgrid} v{variant} step {done}: max|dzs| {dzs:.3g} max|dq| {dq:.3g}")
        assert g.scalars()["nt"] == o.scalars()["nt"]
        assert dzs <= 2e-5 and dq <= 2e-5, (done, dzs, dq)
    g.close()
