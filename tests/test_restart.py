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
    that reaches each output time writes sfincs.<yyyymmdd.HHMMSS of int(t)>.rst
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
        t = g.scalars()["t"]
        s = int(t)
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


def test_quadtree_restart_output_is_refused(tmp_path):
    """Restart files on quadtree meshes are not built: asking for restart
    output there is an error at load, not a file with the fluxes missing."""
    from sfincs_b200 import bmi as B
    from sfincs_b200 import qtsynth

    m = qtsynth.quadtree_coastal(nmax1=6, mmax1=8, dx1=400.0, nlev=2, bands=(600.0,), P=2, seed=4, tstop=600.0,
                                 subgrid=False)
    d = m.write(str(tmp_path))
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'dtrstout':<20} = 300\n")
    with pytest.raises(RuntimeError, match="restart output"):
        B.layout(d, "counts", 10)
