"""GPU parity of the quadtree path: the face/cell kernels on multi-level
meshes against the oracle in the core's precision, step by step, plus lake at
rest, volume balance across refinement levels, and ensemble members alone vs
in the mix."""
import numpy as np
import pytest

from sfincs_b200 import qtsynth
from sfincs_b200.bmi import Ensemble, Model

pytestmark = pytest.mark.gpu


def _oracle(d, prec):
    from oracle.oracle import Oracle

    return Oracle(d, prec)


def _write(tmp_path, subgrid, seed=21, wind=30.0, tstop=1800.0, name="m", edges=False):
    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=seed,
                                 tstop=tstop, subgrid=subgrid, wind_speed=wind, tide_period=1800.0)
    if edges:  # lateral Neumann edges (msk 6) north and south, a downstream river edge (msk 5) east
        lev, n, mm = m.mesh.level, m.mesh.n, m.mesh.m
        nmax_l, mmax_l = 8 * 2 ** (lev - 1), 10 * 2 ** (lev - 1)
        lateral = ((n == 1) | (n == nmax_l)) & (m.mask != 2)
        m.mask[lateral] = 6
        m.mask[(mm == mmax_l) & ~lateral] = 5
    d = tmp_path / name
    d.mkdir()
    out = m.write(str(d))
    if edges:
        import os

        with open(os.path.join(out, "sfincs.bdr"), "w") as f:  # x y x_internal y_internal slope distance
            f.write("3950.0 1600.0 2950.0 1600.0 0.0005 -1.0\n3950.0 500.0 3450.0 700.0 0.0002 600.0\n")
        with open(os.path.join(out, "sfincs.inp"), "a") as f:
            f.write(f"{'bdrfile':<20} = sfincs.bdr\n")
    return out, m


def _cell_q(o, n_cells, npq):
    """Oracle q of each cell's right / upper uv point (combined points and the dummy included)."""
    q = o.get("q", npq)
    qx = q[o.get("z_uv_mu", n_cells).astype(int) - 1]
    qy = q[o.get("z_uv_nu", n_cells).astype(int) - 1]
    return qx, qy


def _add_sources(d):
    """Three point sources (x, y in metres) with a discharge series (m3/s)."""
    import os

    np.savetxt(os.path.join(d, "sfincs.src"), np.array([[1000.0, 1000.0], [2500.0, 1600.0], [3500.0, 2800.0]]),
               fmt="%.4f")
    np.savetxt(os.path.join(d, "sfincs.dis"), np.array([[0.0, 5.0, 0.0, 2.0], [900.0, 20.0, 3.0, 2.0],
                                                        [2000.0, 0.0, 6.0, 2.0]]), fmt="%.6f")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'srcfile':<20} = sfincs.src\n{'disfile':<20} = sfincs.dis\n")


def _add_thin_dams(d):
    """A dam across the domain and a bent one over several refinement levels."""
    import os

    with open(os.path.join(d, "sfincs.thd"), "w") as f:
        f.write("D1\n2 2\n1900.0 -100.0\n2100.0 3300.0\nD2\n3 2\n300.0 2500.0\n1500.0 1500.0\n3900.0 2900.0\n")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'thdfile':<20} = sfincs.thd\n")


def _add_weirs(d):
    """A weir across the domain with a varying crest and one along it."""
    import os

    with open(os.path.join(d, "sfincs.weir"), "w") as f:
        f.write("W1\n3 4\n2300.0 -100.0 -1.0 1.0\n2200.0 1600.0 0.5 0.8\n2400.0 3300.0 1.0 0.9\n"
                "W2\n2 4\n200.0 1700.0 0.5 1.0\n3900.0 1500.0 2.0 1.0\n")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'weirfile':<20} = sfincs.weir\n")


def _add_drainage(d):
    """The five drainage structure types between cells of different levels."""
    import os

    rows = ["500.0 500.0 2500.0 2500.0 1 2.0",
            "900.0 2100.0 3100.0 1700.0 2 1.5",
            "1300.0 2900.0 700.0 1500.0 3 1.0",
            "1700.0 700.0 300.0 2700.0 4 3.0 -6.0 0.02 -3.0 4.0 120.0",
            "2100.0 1300.0 3700.0 300.0 5 2.0 -8.0 0.025 600.0 1500.0 60.0"]
    with open(os.path.join(d, "sfincs.drn"), "w") as f:
        f.write("\n".join(rows) + "\n")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'drnfile':<20} = sfincs.drn\n")


def _add_infiltration(d):
    """A c2d infiltration field (mm/h per cell, cell order) under the rain."""
    import os

    from sfincs_b200 import bmi as B

    n = int(B.layout(d, "qt_counts", 4)[0])
    rng = np.random.default_rng(5)
    rng.uniform(0.0, 20.0, n).astype(np.float32).tofile(os.path.join(d, "sfincs.qinf"))
    np.savetxt(os.path.join(d, "sfincs.prcp"), np.array([[0.0, 30.0], [7200.0, 30.0]]), fmt="%.6f")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'qinffile':<20} = sfincs.qinf\n{'prcfile':<20} = sfincs.prcp\n")


def _add_green_ampt(d):
    """Green-Ampt infiltration (suction head, moisture deficit, conductivity per cell) under rain that stops."""
    import os

    from sfincs_b200 import bmi as B

    n = int(B.layout(d, "qt_counts", 4)[0])
    rng = np.random.default_rng(6)
    for name, lo, hi in (("psi", 50.0, 300.0), ("sigma", 0.1, 0.4), ("ks", 5.0, 20000.0)):
        rng.uniform(lo, hi, n).astype(np.float32).tofile(os.path.join(d, f"sfincs.{name}"))
    np.savetxt(os.path.join(d, "sfincs.prcp"), np.array([[0.0, 40.0], [400.0, 40.0], [401.0, 0.0], [7200.0, 0.0]]),
               fmt="%.6f")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        for key, name in (("psifile", "psi"), ("sigmafile", "sigma"), ("ksfile", "ks"), ("prcfile", "prcp")):
            f.write(f"{key:<20} = sfincs.{name}\n")


@pytest.mark.parametrize("subgrid,extra", [(False, "green_ampt"), (True, "green_ampt"),
                                           (False, "infiltration"), (True, "infiltration"),
                                           (False, None), (True, None), (False, "sources"), (True, "sources"),
                                           (False, "dams"), (True, "dams"), (False, "weirs"), (True, "weirs"),
                                           (False, "drainage"), (True, "drainage"), (False, "edges"),
                                           (True, "edges")])
def test_quadtree_stepwise_matches_f32_oracle(tmp_path, subgrid, extra):
    from sfincs_b200 import bmi as B

    d, _ = _write(tmp_path, subgrid, edges=extra == "edges")
    if extra == "sources":
        _add_sources(d)
    if extra == "drainage":
        _add_drainage(d)
    if extra == "infiltration":
        _add_infiltration(d)
    if extra == "green_ampt":
        _add_green_ampt(d)
    if extra == "weirs":
        _add_weirs(d)
        n = int(_oracle(d, "f32").get("nrstructures", 1)[0])
        assert n > 5 and int(B.layout(d, "nstruc", 1)[0]) == n
    if extra == "dams":
        _add_thin_dams(d)
        qc = B.layout(d, "qt_counts", 4)
        act = B.layout(d, "uv_act", int(qc[1]))
        kc = _oracle(d, "f32").get("kcuv", int(qc[1]))
        assert np.array_equal(act > 0, np.isin(kc, (1, 6)))  # face activity after the dams, face by face
        d0, _ = _write(tmp_path, subgrid, name="open")
        assert int((B.layout(d0, "uv_act", int(qc[1])) > 0).sum()) > int((act > 0).sum())  # the dams removed faces
    qc = B.layout(d, "qt_counts", 4)
    npc, npuv, ncuv = int(qc[0]), int(qc[1]), int(qc[2])
    o = _oracle(d, "f32")
    g = Model(d)
    done = 0
    # The weir discharge switches between free and submerged flow at
    # h2 = 2/3 h1 and stops when both levels fall below the crest: a switch
    # taken one step apart turns an ulp of difference (cube roots and powers
    # are not correctly rounded alike on both sides) into a visible one, so
    # the weir case is compared over the first 40 steps.
    schedule = (1, 1, 2, 6, 30) if extra == "weirs" else (1, 1, 2, 6, 30, 60)
    for n in schedule:
        o.update(-1000.0, n)
        g.step(n)
        done += n
        so, sg = o.scalars(), g.scalars()
        assert sg["nt"] == so["nt"]
        dzs = float(np.abs(g.get("zs") - o.get("zs")).max())
        qx, qy = _cell_q(o, npc, npuv + ncuv + 1)
        dq = max(float(np.abs(g.get("qx") - qx).max()), float(np.abs(g.get("qy") - qy).max()))
        print(f"quadtree subgrid={subgrid} step {done}: dt {so['dt']:.6g}/{sg['dt']:.6g} |dzs| {dzs:.3g} |dq| {dq:.3g}")
        assert dzs <= 2e-5 and dq <= 2e-5, (done, dzs, dq)
        assert abs(sg["t"] - so["t"]) <= 1e-6 * max(1.0, abs(so["t"]))


@pytest.mark.parametrize("subgrid", [False, True])
def test_quadtree_weirs_long_run(tmp_path, subgrid):
    """Past the free/submerged switches: over 600 steps the weir faces keep
    the FP64 volume balance, and the levels stay with the oracle's within a
    bar that a dropped or doubled weir flux would exceed."""
    d, _ = _write(tmp_path, subgrid, tstop=7200.0)
    _add_weirs(d)
    o = _oracle(d, "f32")
    g = Model(d)
    v0 = g.volume()
    for n in (200, 200, 200):
        o.update(-1000.0, n)
        g.step(n)
        s = g.scalars()
        dz = np.abs(g.get("zs") - o.get("zs"))
        print(f"weirs subgrid={subgrid} nt {s['nt']:.0f}: mean|dzs| {dz.mean():.3g} max|dzs| {dz.max():.3g}")
        assert s["nt"] == o.scalars()["nt"]
        assert float(dz.mean()) <= 2e-3 and float(dz.max()) <= 0.1
    v1 = g.volume()
    src = s["bflux_vol"] + s["rain_vol"] + s["src_vol"]
    assert abs((v1 - v0) - src) / max(abs(v1), 1.0) <= 1e-6, (v1 - v0, src)
    g.close()


def test_quadtree_lake_at_rest(tmp_path):
    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=1800.0, subgrid=False, wind_speed=0.0)
    m.mask[:] = 1
    m.bnd = m.bzs = m.wnd = None
    m.z = np.minimum(m.z, -1.0).astype(np.float32)
    m.params["zsini"] = 0.5
    d = m.write(str(tmp_path))
    g = Model(d)
    z0 = g.get("zs")
    g.step(100)
    assert np.array_equal(g.get("zs"), z0)
    assert np.all(g.get("qx") == 0) and np.all(g.get("qy") == 0)


def test_quadtree_volume_balance(tmp_path):
    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=22,
                                 tstop=1800.0, subgrid=True, wind_speed=10.0, tide_period=1800.0)
    m.prcp = np.array([[0.0, 60.0], [7200.0, 60.0]])
    d = m.write(str(tmp_path))
    g = Model(d)
    v0 = g.volume()
    g.step(200)
    s = g.scalars()
    v1 = g.volume()
    src = s["bflux_vol"] + s["rain_vol"] + s["src_vol"]
    assert abs((v1 - v0) - src) / max(abs(v1), 1.0) <= 1e-6, (v1 - v0, src)


def test_quadtree_members_alone_equal_in_mix(tmp_path):
    dirs = [_write(tmp_path, True, seed=30 + i, tstop=900.0 + 300.0 * i, name=f"m{i}")[0] for i in range(3)]
    e = Ensemble(dirs)
    e.run([e.scalars(i)["t1"] for i in range(len(dirs))])
    for i, d in enumerate(dirs):
        g = Model(d)
        g.run(g.scalars()["t1"])
        assert e.scalars(i)["nt"] == g.scalars()["nt"]
        for name in ("zs", "qx", "qy", "zsmax"):
            assert np.array_equal(e.get(i, name), g.get(name)), (i, name)
        g.close()
    e.close()
