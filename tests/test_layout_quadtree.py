"""The CUDA core's quadtree mesh build (host side, no GPU) against the oracle:
uv points, their eight neighbours, combined points, cell-to-uv indices,
advection mask, boundary faces, bed and initial state, on multi-level meshes."""
import numpy as np
import pytest

from sfincs_b200 import bmi as B
from sfincs_b200 import qtsynth


def _oracle(d, prec="f32"):
    from oracle.oracle import Oracle

    return Oracle(d, prec)


def _model(tmp_path, subgrid, seed=21, nlev=3, advection=1, viscosity=1, walk_km=0.0):
    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=nlev, bands=(1000.0, 500.0, 250.0)[: nlev - 1],
                                 P=4, seed=seed, tstop=1800.0, subgrid=subgrid, advection=advection,
                                 viscosity=viscosity, walk_km=walk_km)
    return m.write(str(tmp_path)), m


@pytest.mark.parametrize("subgrid,nlev,walk_km", [(False, 3, 0.0), (True, 3, 0.0), (True, 4, 12.0)])
def test_quadtree_mesh_matches_oracle(tmp_path, subgrid, nlev, walk_km):
    d, m = _model(tmp_path, subgrid, nlev=nlev, walk_km=walk_km)
    o = _oracle(d)
    s = o.scalars()
    qc = B.layout(d, "qt_counts", 4)
    npc, npuv, ncuv = int(qc[0]), int(qc[1]), int(qc[2])
    assert npc == int(s["np"]) and npuv == int(s["npuv"])
    assert ncuv > 0 and int(qc[3]) == nlev
    for name in ("uv_nm", "uv_nmu", "uv_dir", "uv_iref", "uv_u_nmd", "uv_u_nmu", "uv_u_ndm", "uv_u_num",
                 "uv_v_ndm", "uv_v_nm", "uv_v_ndmu", "uv_v_nmu"):
        assert np.array_equal(B.layout(d, name, npuv), o.get(name, npuv)), name
    assert np.array_equal(B.layout(d, "uv_trans", npuv), (o.get("uv_type", npuv) != 0).astype(float))
    for name in ("z_uv_md", "z_uv_mu", "z_uv_nd", "z_uv_nu"):
        assert np.array_equal(B.layout(d, name, npc), o.get(name, npc)), name
    for name in ("cuv_uv1", "cuv_uv2"):
        assert np.array_equal(B.layout(d, name, ncuv), o.get(name, ncuv)), name
    kcuv = o.get("kcuv", npuv)
    assert np.array_equal(B.layout(d, "uv_act", npuv), ((kcuv == 1) | (kcuv == 6)).astype(float))
    assert np.array_equal(B.layout(d, "uv_adv", npuv), o.get("mask_adv", npuv))
    cnt = B.layout(d, "counts", 10)
    nkb = int(cnt[3])
    assert nkb == int(s["nkcuv2"]) and nkb > 0
    for name in ("kb_cell", "kb_dir", "kb_sign"):
        assert np.array_equal(B.layout(d, name, nkb), o.get(name, nkb)), name
    assert np.array_equal(B.layout(d, "zs", npc), o.get("zs"))
    assert float(cnt[6]) == pytest.approx(s["dtmax"], rel=0, abs=0)
    if subgrid:
        assert np.array_equal(B.layout(d, "zvol", npc), o.get("z_volume"))
    else:
        assert np.array_equal(B.layout(d, "zbuvmx", npuv), o.get("zbuvmx", npuv))
        act = kcuv > 0
        assert np.array_equal(B.layout(d, "gn2uv", npuv)[act], o.get("gn2uv", npuv)[act])


@pytest.mark.parametrize("subgrid", [False, True])
def test_quadtree_inifile(tmp_path, subgrid):
    """A binary inifile on a quadtree mesh: levels in sfincs cell order."""
    import os

    d, m = _model(tmp_path, subgrid)
    npc = int(B.layout(d, "qt_counts", 4)[0])
    rng = np.random.default_rng(9)
    rng.uniform(-3.0, 2.0, npc).astype(np.float32).tofile(os.path.join(d, "sfincs.ini"))
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'inifile':<20} = sfincs.ini\n")
    o = _oracle(d)
    zs = B.layout(d, "zs", npc)
    assert np.array_equal(zs, o.get("zs", npc))
    assert np.any(zs != B.layout(_model(tmp_path / "plain", subgrid)[0], "zs", npc))


@pytest.mark.parametrize("subgrid", [False, True])
def test_quadtree_neumann_and_river_edges_match_oracle(tmp_path, subgrid):
    """Lateral Neumann edges (msk 6) and a downstream river edge (msk 5) on a
    3-level mesh: face activity and the water-level boundary faces (river
    faces included, lateral faces left to the momentum kernel) face by face."""
    import sys

    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent))
    from test_gpu_quadtree import _write

    d, m = _write(tmp_path, subgrid, edges=True)
    assert (m.mask == 6).sum() > 10 and (m.mask == 5).sum() > 5
    o = _oracle(d)
    qc = B.layout(d, "qt_counts", 4)
    npc, npuv = int(qc[0]), int(qc[1])
    kcuv = o.get("kcuv", npuv)
    assert (kcuv == 6).sum() > 10
    assert np.array_equal(B.layout(d, "uv_act", npuv), ((kcuv == 1) | (kcuv == 6)).astype(float))
    nkb = int(B.layout(d, "counts", 10)[3])
    # the oracle's list holds kcuv 2 and 6 faces; those of Neumann cells that
    # found a regular neighbour belong to the momentum kernel, isolated ones
    # (reset to inactive) stay in the list with their level at 0; the oracle's
    # getter returns exactly the kept faces and refuses any other length
    assert nkb > int((kcuv == 2).sum())
    for name in ("kb_cell", "kb_dir", "kb_sign"):
        assert np.array_equal(B.layout(d, name, nkb), o.get(name, nkb)), name
