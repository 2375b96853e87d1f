"""Binary restart files (sfincs_initial_conditions.F90:183-268).

A restart file holds Fortran unformatted records framed by their byte
lengths: the flavour, zs (float32[np]), q (float32[npuv + ncuv + 1],
reference face order) and uvmean (float32[nkcuv2]).  These tests write one
from an oracle state, start the oracle and the CUDA core from it, and check
that both start from the file's values and then stay together.
"""
import os
import shutil

import numpy as np
import pytest

from conftest import oracle_faces_to_cells, small_plain, small_subgrid


def write_restart(path, zs, q, uvmean, rsttype=1):
    with open(path, "wb") as f:
        for arr in (np.array([rsttype], np.int32), np.asarray(zs, np.float32), np.asarray(q, np.float32),
                    np.asarray(uvmean, np.float32)):
            b = arr.tobytes()
            n = np.array([len(b)], np.int32).tobytes()
            f.write(n + b + n)


def _restart_dir(tmp_path, make, steps=40):
    """Run the core-precision oracle `steps` steps, write its state as
    sfincs.rst and return a copy of the model directory that starts from it."""
    from oracle.oracle import Oracle

    d, _ = make(tmp_path / "a")
    o = Oracle(d, "f32")
    o.update(-1000.0, steps)
    s = o.scalars()
    zs, q, uvm = o.get("zs"), o.get("q"), o.get("uvmean")
    d2 = str(tmp_path / "b")
    shutil.copytree(d, d2)
    write_restart(os.path.join(d2, "sfincs.rst"), zs, np.append(q, 0.0), uvm)
    with open(os.path.join(d2, "sfincs.inp"), "a") as f:
        f.write(f"{'rstfile':<20} = sfincs.rst\n")
    return d2, zs, q, uvm, int(s["npuv"])


@pytest.mark.parametrize("make", [small_plain, small_subgrid], ids=["plain", "subgrid"])
def test_oracle_starts_from_restart(tmp_path, make):
    from oracle.oracle import Oracle

    d2, zs, q, uvm, npuv = _restart_dir(tmp_path, make)
    o = Oracle(d2, "f32")
    assert np.array_equal(o.get("zs"), zs)  # every level was above the bed already
    assert np.array_equal(o.get("q"), q)
    assert np.array_equal(o.get("uvmean"), uvm)


def test_layout_reads_restart(tmp_path):
    from sfincs_b200 import bmi as B

    d2, zs, q, uvm, npuv = _restart_dir(tmp_path, small_subgrid)
    n = zs.size
    assert np.array_equal(B.layout(d2, "zs", n), zs.astype(np.float32))


def test_bad_restart_is_refused(tmp_path):
    from sfincs_b200 import bmi as B

    d, _ = small_plain(tmp_path)
    write_restart(os.path.join(d, "sfincs.rst"), np.zeros(3), np.zeros(5), np.zeros(2))
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'rstfile':<20} = sfincs.rst\n")
    with pytest.raises(RuntimeError, match="restart"):
        B.layout(d, "counts", 10)


@pytest.mark.gpu
@pytest.mark.parametrize("make", [small_plain, small_subgrid], ids=["plain", "subgrid"])
def test_gpu_continues_from_restart_with_oracle(tmp_path, make):
    """The core started from a restart file holds the file's state and then
    matches the oracle started from the same file, step by step."""
    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model

    d2, zs, q, uvm, npuv = _restart_dir(tmp_path, make)
    o = Oracle(d2, "f32")
    g = Model(d2)
    assert np.array_equal(g.get("zs").astype(np.float64), zs)
    qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
    assert np.array_equal(g.get("qx"), qx_o) and np.array_equal(g.get("qy"), qy_o)
    done = 0
    for n in (1, 1, 2, 6, 30):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        so, sg = o.scalars(), g.scalars()
        dzs = float(np.abs(o.get("zs") - g.get("zs")).max())
        qx_o, qy_o = oracle_faces_to_cells(o, o.get("q"))
        dq = max(float(np.abs(qx_o - g.get("qx")).max()), float(np.abs(qy_o - g.get("qy")).max()))
        assert sg["nt"] == so["nt"]
        assert abs(sg["t"] - so["t"]) <= 1e-6 * max(1.0, abs(so["t"]))
        assert dzs <= 2e-5, f"zs differs by {dzs} after {done} steps"
        assert dq <= 2e-5, f"q differs by {dq} after {done} steps"
    g.close()


def read_restart(path):
    recs = []
    with open(path, "rb") as f:
        while True:
            head = f.read(4)
            if not head:
                break
            n = int(np.frombuffer(head, np.int32)[0])
            recs.append(f.read(n))
            assert int(np.frombuffer(f.read(4), np.int32)[0]) == n
    return (int(np.frombuffer(recs[0], np.int32)[0]),) + tuple(np.frombuffer(r, np.float32) for r in recs[1:])


@pytest.mark.gpu
def test_gpu_writes_restart_files_at_output_times(tmp_path):
    """dtrstout (sfincs_output.f90:657-733, sfincs_lib.f90:447-463): the step
    that reaches each output time writes sfincs.<yyyymmdd.HHMMSS of the output time>.rst
    with that step's zs, q (reference face order) and uvmean; a model started
    from the file holds the same state."""
    import glob

    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model

    d, _ = small_subgrid(tmp_path)
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'dtrstout':<20} = 600\n")
    o = Oracle(d, "f32")
    cell = o.get("uv_nm").astype(np.int64) - 1
    dirn = o.get("uv_dir").astype(np.int64)
    g = Model(d)
    seen = set()
    checked = 0
    while g.scalars()["t"] < 1900.0:
        g.step(1)
        new = set(glob.glob(os.path.join(d, "sfincs.*.rst"))) - seen
        if not new:
            continue
        assert len(new) == 1
        path = new.pop()
        seen.add(path)
        s = 600 * (checked + 1)  # named from the output time, not the step's end (sfincs_lib.f90:447-463)
        assert g.scalars()["t"] >= s
        assert os.path.basename(path) == f"sfincs.20000101.{s // 3600:02d}{s % 3600 // 60:02d}{s % 60:02d}.rst"
        typ, zs, q, uvm = read_restart(path)
        assert typ == 1
        assert np.array_equal(zs, g.get("zs").astype(np.float32))
        qx, qy = g.get("qx"), g.get("qy")
        assert q.size == cell.size + 1 and q[-1] == 0.0
        assert np.array_equal(q[:-1], np.where(dirn == 0, qx[cell], qy[cell]).astype(np.float32))
        d2 = str(tmp_path / f"from{checked}")
        shutil.copytree(d, d2)
        with open(os.path.join(d2, "sfincs.inp"), "a") as f:
            f.write(f"{'rstfile':<20} = {os.path.basename(path)}\n")
        g2 = Model(d2)
        assert np.array_equal(g2.get("zs"), g.get("zs"))
        g2.close()
        checked += 1
    assert checked == 3  # 600, 1200 and 1800 s
    g.close()


def _qt_restart_dirs(tmp_path, subgrid, steps=40):
    """A 3-level quadtree model, its oracle state after `steps` steps written
    as a restart file, and a copy of the model that starts from it."""
    from oracle.oracle import Oracle
    from sfincs_b200 import bmi as B
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                 tstop=1800.0, subgrid=subgrid, wind_speed=30.0, tide_period=1800.0)
    d = m.write(str(tmp_path / "a"))
    qc = B.layout(d, "qt_counts", 4)
    npc, npuv, ncuv = int(qc[0]), int(qc[1]), int(qc[2])
    o = Oracle(d, "f32")
    o.update(-1000.0, steps)
    zs, q, uvm = o.get("zs", npc), o.get("q", npuv + ncuv + 1), o.get("uvmean")
    d2 = str(tmp_path / "b")
    shutil.copytree(d, d2)
    write_restart(os.path.join(d2, "sfincs.rst"), zs, q, uvm)
    with open(os.path.join(d2, "sfincs.inp"), "a") as f:
        f.write(f"{'rstfile':<20} = sfincs.rst\n")
    return d, d2, zs, q, npc, npuv, ncuv


@pytest.mark.parametrize("subgrid", [False, True])
def test_quadtree_restart_is_read(tmp_path, subgrid):
    """Quadtree restart files: zs per cell and q per uv point in the
    reference's order; the oracle and the core's layout start from them."""
    from oracle.oracle import Oracle
    from sfincs_b200 import bmi as B

    d, d2, zs, q, npc, npuv, ncuv = _qt_restart_dirs(tmp_path, subgrid)
    o = Oracle(d2, "f32")
    assert np.array_equal(o.get("zs", npc), zs)
    assert np.array_equal(o.get("q", npuv), q[:npuv])
    assert np.array_equal(B.layout(d2, "zs", npc), zs)


@pytest.mark.gpu
@pytest.mark.parametrize("subgrid", [False, True])
def test_gpu_quadtree_restart_round_trip(tmp_path, subgrid):
    """The core started from a quadtree restart file follows the oracle started
    from it, and the file the core writes (dtrstout) holds its own state in the
    reference's order and length."""
    import glob

    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model

    d, d2, zs, q, npc, npuv, ncuv = _qt_restart_dirs(tmp_path, subgrid)
    o = Oracle(d2, "f32")
    g = Model(d2)
    assert np.array_equal(g.get("zs").astype(np.float64), zs)
    done = 0
    for n in (1, 1, 2, 6, 30):
        o.update(-1000.0, n)
        g.step(n)
        done += n
        dzs = float(np.abs(o.get("zs", npc) - g.get("zs")).max())
        assert g.scalars()["nt"] == o.scalars()["nt"]
        assert dzs <= 2e-5, (done, dzs)
    g.close()
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'dtrstout':<20} = 600\n")
    g = Model(d)
    files = []
    while not files and g.scalars()["t"] < 900.0:
        g.step(1)
        files = sorted(glob.glob(os.path.join(d, "sfincs.*.rst")))
    zs_now = g.get("zs").astype(np.float32)
    g.close()
    assert files
    typ, zs_f, q_f, uvm_f = read_restart(files[0])
    assert typ == 1 and zs_f.size == npc and q_f.size == npuv + ncuv + 1
    assert np.array_equal(zs_f, zs_now)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,flavour", [("cnb", 4), ("gai", 5), ("hor", 6)])
def test_gpu_restart_flavours_with_infiltration_state(tmp_path, kind, flavour):
    """With a curve-number-with-recovery, Green-Ampt or Horton model the
    restart file is flavour 4, 5 or 6 and carries that method's state
    (sfincs_output.f90:690-722); the core and the oracle started from it stay
    together step by step."""
    import glob

    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model
    from test_gpu_physics import _infiltration_fields, _plain, _subgrid

    m = (_subgrid if kind == "hor" else _plain)(tmp_path, dtrstout=600)
    d = _infiltration_fields(m, kind).write(str(tmp_path / "a"))
    g = Model(d)
    g.run(650.0)
    g.close()
    files = sorted(glob.glob(os.path.join(d, "sfincs.*.rst")))
    assert files, "no restart file written"
    recs = read_restart(files[0])
    assert recs[0] == flavour
    n = recs[1].size
    assert len(recs) == (6 if flavour == 5 else 5) and all(r.size == n for r in recs[4:])
    d2 = str(tmp_path / "b")
    shutil.copytree(d, d2)
    with open(os.path.join(d2, "sfincs.inp"), "a") as f:
        f.write(f"{'rstfile':<20} = {os.path.basename(files[0])}\n")
    o = Oracle(d2, "f32")
    g = Model(d2)
    done = 0
    for k in (1, 5, 30, 60):
        o.update(-1000.0, k)
        g.step(k)
        done += k
        dzs = float(np.abs(o.get("zs") - g.get("zs")).max())
        assert g.scalars()["nt"] == o.scalars()["nt"]
        assert dzs <= 2e-5, (done, dzs)
    g.close()
