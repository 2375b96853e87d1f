"""Map, his and max output (sfincs_output.f90:8-296, sfincs_ncoutput.F90:
148-1590): the files the core writes off the step's critical path hold, at
the reference's output times, the state the oracle has after the step that
reaches each time; the max fields restart after every max output."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FILL = -99999.0


def _nc(path):
    from scipy.io import netcdf_file

    f = netcdf_file(path, "r", mmap=False)
    return f


def _model(tmp_path, extra, quadtree=False, subgrid=False, crs=True, drn=False):
    from crs_cases import add_crs
    from sfincs_b200 import qtsynth, synth

    if quadtree:
        m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                     tstop=3600.0, subgrid=subgrid, wind_speed=10.0, tide_period=1800.0)
    elif subgrid:
        m = synth.subgrid_regular(nmax=20, mmax=24, dx=500.0, P=8, seed=5, tstop=3600.0, rain_mmh=40.0,
                                  rain_hours=0.5, coast_x=24 * 500.0 * 0.3, t_peak=1800.0, width_h=0.5,
                                  surge_peak=1.5)
    else:
        m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=3600.0, seed=3, nbumps=6)
    if drn:  # the five drainage structure types
        from test_gpu_physics import _DRAINAGE

        m.drn = _DRAINAGE
    d = m.write(str(tmp_path))
    with open(os.path.join(d, "sfincs.obs"), "w") as f:
        f.write("1000.0 1000.0 'harbour'\n2600.0 1800.0\n-500.0 -500.0 \"outside\"\n")
    keys = dict(obsfile="sfincs.obs")
    keys.update(extra)
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        for k, v in keys.items():
            f.write(f"{k:<20} = {v}\n")
    if crs:  # three cross-sections (the quadtree mesh spans 4 km x 3.2 km)
        add_crs(d, scale=1.0 / 3.0 if quadtree else 1.0)
    if drn:  # two run-up gauges from the sea onto the beach
        with open(os.path.join(d, "sfincs.rug"), "w") as f:
            f.write("rug_south\n2 2\n500.0 3000.0\n11000.0 3000.0\nrug_north\n2 2\n500.0 7000.0\n11000.0 7000.0\n")
        with open(os.path.join(d, "sfincs.inp"), "a") as f:
            f.write(f"{'rugfile':<20} = sfincs.rug\n{'rugdepth':<20} = 0.05\n")
    return d, m


class Expected:
    """The oracle stepped one step at a time, with the reference's output
    schedule (sfincs_lib.f90:419-476): per output, its time and the state."""

    def __init__(self, d, dtmap, dthis, dtmax, stored=("vmax_out", "twet_out"), ncrs=3, ndrn=0, nrug=0):
        from oracle.oracle import Oracle

        self.stored = stored
        self.o = o = Oracle(d, "f32")
        s = o.scalars()
        self.np = n = int(s["np"])
        t0, t1 = s["t0"], s["t1"]
        self.zb = o.get("z_zmin") if s["subgrid"] else o.get("zb")
        md, mu = o.get("z_uv_md", n).astype(np.int64), o.get("z_uv_mu", n).astype(np.int64)
        nd, nu = o.get("z_uv_nd", n).astype(np.int64), o.get("z_uv_nu", n).astype(np.int64)
        self.map, self.his, self.max, self.crs, self.drn, self.rug = [], [], [], [], [], []
        tmap, this, tmax = t0, t0, t0 + dtmax
        nmax_before = 0
        while o.scalars()["t"] < t1:
            o.update(-1000.0, 1)
            s = o.scalars()
            t, dt = s["t"], s["dt"]
            wmap = wmax = whis = False
            tout = t
            if t >= tmap:
                wmap, tout = True, max(tmap, t - dt)
                tmap += dtmap
            if t >= tmax:
                wmax, tout = True, max(tmax, t - dt)
                if t < t1:
                    tmax += dtmax
            if t >= this:
                whis, tout = True, max(this, t - dt)
                this += dthis
            zs = o.get("zs").astype(np.float32)
            uv = np.concatenate([[0.0], o.get("uv"), [0.0]])  # 1-based; 0 and npuv + 1 (the dummy) hold 0
            u = (0.5 * uv[md] + 0.5 * uv[mu]).astype(np.float32)
            v = (0.5 * uv[nd] + 0.5 * uv[nu]).astype(np.float32)
            if wmap:
                self.map.append((np.float32(tout), zs, u, v))
            if whis:
                self.his.append((np.float32(tout), zs.copy()))
                if ncrs:
                    self.crs.append(o.get("crs_discharge", ncrs))
                if ndrn:
                    self.drn.append(o.get("q_drain", ndrn))
                if nrug:
                    self.rug.append(o.get("runup_zs", nrug))
            if wmax:
                assert int(o.get("ntmaxout", 1)[0]) == nmax_before + 1
                nmax_before += 1
                opt = lambda k: o.get(k) if k in self.stored else None  # noqa: E731
                self.max.append((np.float32(tout), o.get("zsmax_out"), opt("vmax_out"), opt("twet_out")))
        self.t_end = o.scalars()["t"]


@pytest.mark.parametrize("subgrid", [False, True])
def test_netcdf_map_his_and_max_match_the_oracle(tmp_path, subgrid):
    from sfincs_b200.bmi import Model

    extra = dict(dtout=600, dtmaxout=1200, dthisout=300, storevel=1, storevelmax=1, storetwet=1)
    d, m = _model(tmp_path, extra, subgrid=subgrid, drn=True)
    g = Model(d)
    s = g.scalars()
    g.run(s["t1"])
    g.finalize()
    e = Expected(d, 600.0, 300.0, 1200.0, ndrn=5, nrug=2)
    g.close()
    n = e.np
    # map file: cells on the (n, m) grid
    f = _nc(os.path.join(d, "sfincs_map.nc"))
    nmax, mmax = m.msk.shape
    assert f.dimensions["n"] == nmax and f.dimensions["m"] == mmax
    mi, ni = np.nonzero(m.msk.T > 0)  # compact order: n fastest
    zs_f = f.variables["zs"][:]
    assert zs_f.shape[0] == len(e.map) >= 6
    huthresh = 0.0 if subgrid else float(m.params.get("huthresh", 0.05))  # netCDF subgrid tables force 0
    for k, (t, zs, u, v) in enumerate(e.map):
        assert f.variables["time"][k] == t
        got = zs_f[k][ni, mi]
        wet = (zs - e.zb.astype(np.float32)) > huthresh
        assert np.all(got[~wet] == FILL)
        assert np.allclose(got[wet], zs[wet], atol=2e-5), k
        assert np.allclose(f.variables["u"][k][ni, mi], u, atol=2e-5)
        assert np.allclose(f.variables["v"][k][ni, mi], v, atol=2e-5)
        if not subgrid:
            assert np.allclose(f.variables["h"][k][ni, mi], zs - e.zb.astype(np.float32), atol=2e-5)
    inactive = m.msk == 0
    assert np.all(zs_f[0][inactive] == FILL)
    assert np.array_equal(f.variables["msk"][:][m.msk > 0], m.msk[m.msk > 0].astype(np.int32))
    # max: three intervals of 1200 s, each restarted
    assert len(e.max) == 3 and f.dimensions["timemax"] == 3
    for k, (t, zsmax, vmax, twet) in enumerate(e.max):
        assert f.variables["timemax"][k] == t
        got = f.variables["zsmax"][k][ni, mi]
        wet = (zsmax - e.zb) > huthresh
        assert np.all(got[~wet] == FILL)
        assert np.allclose(got[wet], zsmax[wet], atol=2e-5), k
        assert np.allclose(f.variables["vmax"][k][ni, mi], vmax, atol=2e-5)
        assert np.allclose(f.variables["tmax"][k][ni, mi], twet, atol=1e-3)
    assert not np.array_equal(e.max[0][1], e.max[2][1])  # restarted, not cumulative
    assert f.variables["status"][0] == 0.0
    f.close()
    # his file: the two stations inside, the third outside
    h = _nc(os.path.join(d, "sfincs_his.nc"))
    names = [b"".join(r).decode().strip() for r in h.variables["station_name"][:]]
    assert names == ["harbour", "station_002", "outside"]
    cells = [c - 1 for c in _cells(m, [(1000.0, 1000.0), (2600.0, 1800.0), (-500.0, -500.0)])]
    assert cells[2] == -1
    pz = h.variables["point_zs"][:]
    assert pz.shape == (len(e.his), 3)
    for k, (t, zs) in enumerate(e.his):
        assert h.variables["time"][k] == t
        assert np.allclose(pz[k, :2], zs[cells[:2]], atol=2e-5)
        assert pz[k, 2] == FILL
    assert np.allclose(h.variables["point_zb"][:2], e.zb[cells[:2]].astype(np.float32))
    # cross-sections: names and discharges at every his time (sfincs_crosssections.f90:130-176)
    from crs_cases import NAMES

    assert [b"".join(r).decode().strip() for r in h.variables["crosssection_name"][:]] == NAMES
    qd = h.variables["crosssection_discharge"][:]
    assert qd.shape == (len(e.his), 3)
    want = np.array(e.crs)
    assert np.abs(want).max() > 1.0
    assert np.allclose(qd, want, rtol=1e-4, atol=0.2), np.abs(qd - want).max()
    # drainage structures: the rate of each intake at every his time (sfincs_ncoutput.F90:1410-1421)
    qdr = h.variables["drainage_discharge"][:]
    assert qdr.shape == (len(e.his), 5)
    assert np.abs(np.array(e.drn)).max() > 0.1
    assert np.allclose(qdr, np.array(e.drn), rtol=1e-3, atol=1e-3), np.abs(qdr - np.array(e.drn)).max()
    # run-up gauges: the level of the last point wetter than rugdepth (sfincs_runup_gauges.f90:117-150)
    assert [b"".join(r).decode().strip() for r in h.variables["runup_gauge_name"][:]] == ["rug_south", "rug_north"]
    zru, want = h.variables["runup_gauge_zs"][:], np.array(e.rug)
    assert zru.shape == (len(e.his), 2) and np.all(want > -999.0)
    assert np.allclose(zru, want, atol=0.05), np.abs(zru - want).max()
    assert np.mean(np.abs(zru - want) <= 2e-5) >= 0.8
    h.close()


def _cells(m, pts):
    """1-based compact cells of points on an unrotated regular grid (0 outside)."""
    mi, ni = np.nonzero(m.msk.T > 0)
    out = []
    for x, y in pts:
        mm, nn = int(x // m.dx), int(y // m.dy)
        hit = np.nonzero((mi == mm) & (ni == nn))[0] if x >= 0 and y >= 0 else []
        out.append(int(hit[0]) + 1 if len(hit) else 0)
    return out


def test_binary_map_max_and_text_his(tmp_path):
    """outputformat = bin: zs.dat (real*8 records), zsmax.dat (real*4, dry
    cells -999) and zst.txt (f12.1, f9.3) as the reference's binary writers
    lay them out (sfincs_output.f90:298-620)."""
    from sfincs_b200.bmi import Model

    d, m = _model(tmp_path, dict(outputformat="bin", dtout=900, dtmaxout=1800, dthisout=600))
    g = Model(d)
    g.run(g.scalars()["t1"])
    g.finalize()
    g.close()
    e = Expected(d, 900.0, 600.0, 1800.0, stored=())
    n = e.np
    raw = np.fromfile(os.path.join(d, "zs.dat"), np.uint8)
    rec = 4 + 8 * n + 4
    assert raw.size == rec * len(e.map)
    for k, (t, zs, u, v) in enumerate(e.map):
        r = raw[k * rec:(k + 1) * rec]
        assert np.frombuffer(r[:4].tobytes(), np.int32)[0] == 8 * n
        got = np.frombuffer(r[4:-4].tobytes(), np.float64)
        assert np.allclose(got, zs, atol=2e-5)
    raw = np.fromfile(os.path.join(d, "zsmax.dat"), np.uint8)
    rec = 4 + 4 * n + 4
    assert raw.size == rec * len(e.max)
    for k, (t, zsmax, vmax, twet) in enumerate(e.max):
        got = np.frombuffer(raw[k * rec + 4:(k + 1) * rec - 4].tobytes(), np.float32)
        want = np.where(zsmax < e.zb + float(m.params.get("huthresh", 0.05)), -999.0, zsmax)
        assert np.allclose(got, want, atol=2e-5)
    lines = open(os.path.join(d, "zst.txt")).read().splitlines()
    assert len(lines) == len(e.his)
    qt = open(os.path.join(d, "qt.txt")).read().splitlines()
    assert len(qt) == len(e.his)
    for line, want in zip(qt, e.crs):
        assert len(line) == 12 + 12 * 3
        assert np.allclose([float(line[12 + 12 * k:24 + 12 * k]) for k in range(3)], want, rtol=1e-4, atol=0.2)
    for line, (t, zs) in zip(lines, e.his):
        assert len(line) == 12 + 9 * 3
        assert float(line[:12]) == pytest.approx(float(t), abs=0.05)
        assert float(line[12 + 18:]) == -999.0


def test_quadtree_map_file_is_a_ugrid_mesh(tmp_path):
    from sfincs_b200.bmi import Model

    d, m = _model(tmp_path, dict(dtout=1200, dtmaxout=3600, dthisout=600), quadtree=True, subgrid=True)
    g = Model(d)
    g.run(g.scalars()["t1"])
    zs_end = g.get("zs")
    g.finalize()
    g.close()
    f = _nc(os.path.join(d, "sfincs_map.nc"))
    nq = f.dimensions["nmesh2d_face"]
    assert f.dimensions["nmesh2d_node"] == 4 * nq
    fn = f.variables["mesh2d_face_nodes"][:]
    assert fn.shape == (nq, 4) and fn[0, 0] == 1 and fn[-1, 3] == 4 * nq
    assert f.variables["mesh2d"].cf_role == b"mesh_topology"
    msk = f.variables["msk"][:]
    act = msk > 0
    assert act.sum() == zs_end.size
    zs = f.variables["zs"][:]
    assert zs.shape == (4, nq)  # t = 0, 1200, 2400, 3600
    assert np.all(zs[:, ~act] == FILL)
    fx, fy = f.variables["mesh2d_face_x"][:], f.variables["mesh2d_face_y"][:]
    nx = f.variables["mesh2d_node_x"][:].reshape(nq, 4)
    assert np.allclose(fx, nx.mean(axis=1), atol=1e-3)
    assert f.variables["zsmax"][:].shape == (1, nq)
    f.close()
    h = _nc(os.path.join(d, "sfincs_his.nc"))
    qd = h.variables["crosssection_discharge"][:]
    assert qd.shape == (7, 3) and np.all(np.isfinite(qd)) and np.abs(qd).max() > 0.0  # t = 0, 600, ..., 3600
    h.close()
