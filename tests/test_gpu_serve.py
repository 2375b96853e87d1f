"""Serving pool and continuous-batching loop: admission by slots and HBM
budget, requests joining while others run, and every result the same alone
and in the mix (bitwise)."""
import numpy as np
import pytest

from sfincs_b200.bmi import Model
from sfincs_b200.serve import Pool, Prepared, Request, Server

pytestmark = pytest.mark.gpu


def _dirs(tmp_path, n=4):
    from sfincs_b200 import synth

    spec = [(16, 20, 1800.0, 1.0, 60.0), (24, 30, 2400.0, 2.5, 0.0), (40, 28, 1200.0, 3.5, 20.0),
            (20, 36, 3000.0, 2.0, 40.0)]
    dirs = []
    for i, (n_, m, tstop, peak, rain) in enumerate(spec[:n]):
        d = tmp_path / f"r{i}"
        d.mkdir()
        mdl = synth.subgrid_regular(nmax=n_, mmax=m, dx=400.0, P=6, seed=31 + i, tstop=tstop, surge_peak=peak,
                                    rain_mmh=rain, rain_hours=0.25, coast_x=m * 400.0 * 0.3, t_peak=tstop / 2,
                                    width_h=0.3)
        dirs.append(mdl.write(str(d)))
    return dirs


def _alone(d):
    g = Model(d)
    g.run(g.scalars()["t1"])
    out = {k: g.get(k) for k in ("zs", "zsmax", "qx", "qy")}
    out["nt"] = int(g.scalars()["nt"])
    g.close()
    return out


def test_pool_admission_by_slots_and_budget(tmp_path):
    dirs = _dirs(tmp_path, 3)
    preps = [Prepared(d) for d in dirs]
    b = [p.bytes for p in preps]
    assert all(x > 0 for x in b)
    pool = Pool(max_slots=2, hbm_budget_bytes=b[0] + b[1] + 1)
    k0 = pool.admit(preps[0], -1.0)
    k1 = pool.admit(preps[1], -1.0)
    assert k0 >= 0 and k1 >= 0 and k0 != k1
    assert pool.used_bytes == b[0] + b[1]
    assert pool.admit(preps[2], -1.0) == -1  # no slot, no budget: stays with the caller
    pool.release(k0)
    assert pool.used_bytes == b[1]
    if b[2] <= b[0] + 1:
        assert pool.admit(preps[2], -1.0) >= 0
    pool.close()


def test_served_results_equal_alone(tmp_path):
    dirs = _dirs(tmp_path, 4)
    alone = [_alone(d) for d in dirs]
    preps = [Prepared(d) for d in dirs]
    budget = sum(sorted(p.bytes for p in preps)[-2:]) + 1  # at most two requests resident at a time
    for p in preps:
        p.release()
    srv = Server(max_slots=3, hbm_budget_bytes=budget, chunk=8, prep_threads=2)
    reqs = [Request(arrival_s=a, model_dir=d, rid=i) for i, (a, d) in enumerate(zip([0.0, 0.0, 0.02, 0.05], dirs))]
    out = srv.serve(reqs, fetch=("zs", "zsmax", "qx", "qy"))
    srv.close()
    assert len(out["results"]) == 4
    for r in out["results"]:
        a = alone[r.rid]
        assert r.steps == a["nt"], (r.rid, r.steps, a["nt"])
        for k in ("zs", "zsmax", "qx", "qy"):
            assert np.array_equal(r.fields[k], a[k]), (r.rid, k)
        assert r.latency_s >= 0 and r.done_s >= r.admitted_s >= r.arrival_s - 1e-9
    assert out["latency_p99_s"] >= out["latency_p50_s"] > 0
    assert out["mean_running"] > 1.0  # requests really overlapped on the device


def test_served_mix_of_regular_and_quadtree_equals_alone(tmp_path):
    """Regular grids and quadtree meshes in one stream: the pool advances them
    in two runners on two streams, and every result is bitwise the result of
    the same request alone."""
    from sfincs_b200 import qtsynth

    dirs = _dirs(tmp_path, 3)
    for i in range(2):
        m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=40 + i,
                                     tstop=1500.0 + 600.0 * i, subgrid=i == 1, wind_speed=20.0, tide_period=1800.0)
        d = tmp_path / f"q{i}"
        d.mkdir()
        dirs.append(m.write(str(d)))
    alone = [_alone(d) for d in dirs]
    srv = Server(max_slots=4, chunk=8, prep_threads=2)
    arr = [0.0, 0.0, 0.03, 0.0, 0.02]
    reqs = [Request(arrival_s=a, model_dir=d, rid=i) for i, (a, d) in enumerate(zip(arr, dirs))]
    out = srv.serve(reqs, fetch=("zs", "zsmax", "qx", "qy"))
    srv.close()
    assert len(out["results"]) == 5
    for r in out["results"]:
        a = alone[r.rid]
        assert r.steps == a["nt"], (r.rid, r.steps, a["nt"])
        for k in ("zs", "zsmax", "qx", "qy"):
            assert np.array_equal(r.fields[k], a[k]), (r.rid, k)
    assert out["mean_running"] > 1.0
