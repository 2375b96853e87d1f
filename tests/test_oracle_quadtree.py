"""Pins of the oracle's quadtree path (netCDF quadtree files, refinement
transitions, combined uv points).

(1) A single-level quadtree file is the same mesh as the regular index-file
model: the reference reverts to the regular code path (sfincs_domain.f90:42-50)
and the results must be bitwise identical.  (2) Lake at rest and (3) volume
conservation on multi-level meshes, where fluxes cross coarse/fine interfaces
through combined uv points.
"""
import numpy as np
import pytest

from sfincs_b200 import qtsynth, synth


def _oracle(d, prec):
    from oracle.oracle import Oracle

    return Oracle(d, prec)


def _single_level_twin(m: synth.RegularModel, d: str) -> str:
    """Write regular model m again as a one-level quadtree netCDF model."""
    nmax, mmax = m.msk.shape
    lev = np.ones((nmax, mmax), np.int8)
    mesh = qtsynth.build_mesh(lev, nmax, mmax, m.dx, 1)
    mesh.x0, mesh.y0 = m.x0, m.y0
    mask = m.msk.ravel(order="F").astype(np.int8)
    z = (m.zb if m.zb is not None else np.zeros_like(m.msk, np.float32)).ravel(order="F").astype(np.float32)
    qm = qtsynth.QuadtreeModel(mesh=mesh, mask=mask, z=z, sbg=m.sbg, params=dict(m.params), bnd=m.bnd, bzs=m.bzs,
                               prcp=m.prcp, wnd=m.wnd)
    return qm.write(d)


@pytest.mark.parametrize("kind", ["plain", "subgrid"])
def test_single_level_quadtree_equals_regular(tmp_path, kind):
    if kind == "plain":
        m = synth.plain_regular(nmax=10, mmax=14, dx=300.0, tstop=1800.0, seed=4, nbumps=4)
    else:
        m = synth.subgrid_regular(nmax=10, mmax=12, dx=400.0, P=6, seed=8, tstop=1800.0, surge_peak=1.5,
                                  rain_mmh=30.0, rain_hours=0.2, coast_x=1500.0, t_peak=900.0, width_h=0.3)
    (tmp_path / "reg").mkdir()
    (tmp_path / "qt").mkdir()
    dr = m.write(str(tmp_path / "reg"))
    dq = _single_level_twin(m, str(tmp_path / "qt"))
    a, b = _oracle(dr, "ref"), _oracle(dq, "ref")
    assert a.scalars()["np"] == b.scalars()["np"] and a.scalars()["npuv"] == b.scalars()["npuv"]
    a.update(-1000.0, 120)
    b.update(-1000.0, 120)
    assert a.scalars()["t"] == b.scalars()["t"]
    for name in ("zs", "q", "uv", "zsmax"):
        assert np.array_equal(a.get(name), b.get(name)), name


def _closed_quadtree(subgrid, rain=0.0, zsini=0.0, deep=False):
    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=1800.0, subgrid=subgrid, wind_speed=0.0)
    m.mask[:] = 1  # no open boundary
    m.bnd = m.bzs = None
    m.wnd = None
    if deep:
        m.z = np.minimum(m.z, -1.0).astype(np.float32)
    m.params["zsini"] = zsini
    if rain > 0:
        m.prcp = np.array([[0.0, rain], [7200.0, rain]])
    return m


@pytest.mark.parametrize("prec", ["fp64", "ref", "f32"])
def test_quadtree_lake_at_rest(tmp_path, prec):
    m = _closed_quadtree(subgrid=False, zsini=0.5, deep=True)
    assert len(set(m.mesh.level.tolist())) == 3
    d = m.write(str(tmp_path))
    o = _oracle(d, prec)
    z0 = o.get("zs").copy()
    o.update(-1000.0, 100)
    assert np.array_equal(o.get("zs"), z0)
    assert np.all(o.get("q") == 0.0)


def test_quadtree_rain_volume_balance(tmp_path):
    """Closed multi-level subgrid basin under uniform rain: the FP64 volume
    grows by exactly rain x area x time (coarse/fine fluxes cancel)."""
    rain = 50.0
    m = _closed_quadtree(subgrid=True, rain=rain)
    d = m.write(str(tmp_path))
    o = _oracle(d, "ref")
    lev = m.mesh.level[np.nonzero(m.mask > 0)[0]]
    area = float(np.sum((400.0 / 2.0 ** (lev - 1)) ** 2))
    v0 = float(np.sum(o.get("z_volume")))
    o.update(-1000.0, 150)
    s = o.scalars()
    v1 = float(np.sum(o.get("z_volume")))
    expect = np.float32(rain) / np.float32(3.6e6) * area * (s["t"] - s["t0"])
    assert abs((v1 - v0) - expect) <= 2e-6 * max(abs(v1), 1.0), (v1 - v0, expect)
    # flow crossed refinement levels
    assert np.abs(o.get("q")).max() > 0
