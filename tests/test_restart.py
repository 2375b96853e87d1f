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
