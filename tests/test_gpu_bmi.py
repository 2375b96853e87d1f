"""GPU tests of the reference BMI surface (sfincs_bmi.f90) through the C-ABI.

A coupler drives the model with initialize / update / update_until and reads
and writes the arrays that get_value_ptr exports: qext (float, written by the
coupler before each update) and zs (double, refreshed by every update).  The
handle API (sfg_model_*) drives a second copy of the same model with the same
source terms set synchronously before each step; both must hold the same bits
after every step.  update() pushes the exported qext on a side stream while the
step's boundary and momentum kernels run, so these tests also pin that the
continuity kernel sees the new qext of its own step.
"""
import numpy as np
import pytest

from conftest import small_plain, small_subgrid

pytestmark = pytest.mark.gpu

CASES = {"plain": small_plain, "subgrid": small_subgrid}


def _pair(d):
    from sfincs_b200.bmi import BMI, Model

    b = BMI()
    b.initialize(d)
    return b, Model(d, bmi=True)


@pytest.mark.parametrize("kind", sorted(CASES))
def test_update_with_exported_qext_matches_handle_api(tmp_path, kind):
    d, _ = CASES[kind](tmp_path)
    b, g = _pair(d)
    try:
        q = b.get_value_ptr("qext")
        zs = b.get_value_ptr("zs")
        assert q.dtype == np.float32 and zs.dtype == np.float64 and q.size == zs.size == g.np
        rng = np.random.default_rng(4)
        for k in range(40):
            v = rng.uniform(-2.0e-5, 5.0e-5, q.size).astype(np.float32)  # m/s, new every step
            q[:] = v
            b.update()
            g.set("qext", v)
            g.step(1)
            assert np.array_equal(zs, g.get("zs").astype(np.float64)), f"zs differs after update {k + 1}"
        assert b.get_current_time() == pytest.approx(g.scalars()["t"], rel=0, abs=1e-9)
    finally:
        g.close()
        b.finalize()


def test_update_until_matches_handle_api(tmp_path):
    d, _ = small_subgrid(tmp_path)
    b, g = _pair(d)
    try:
        q = b.get_value_ptr("qext")
        zs = b.get_value_ptr("zs")
        q[:] = 1.0e-5
        g.set("qext", np.full(g.np, 1.0e-5, np.float32))
        t_target = b.get_start_time() + 0.5 * (b.get_end_time() - b.get_start_time())
        b.update_until(t_target)
        g.run(t_target)
        assert np.array_equal(zs, g.get("zs").astype(np.float64))
        assert b.get_current_time() >= t_target
    finally:
        g.close()
        b.finalize()


def test_qext_pointer_changes_the_next_step_only(tmp_path):
    """A source term written after update() acts on the following step: the
    level rises by qext * dt there, not before."""
    d, _ = small_plain(tmp_path)
    b, g = _pair(d)
    try:
        q = b.get_value_ptr("qext")
        zs = b.get_value_ptr("zs")
        for _ in range(5):
            b.update()
            g.step(1)
        before = zs.copy()
        assert np.array_equal(before, g.get("zs").astype(np.float64))
        q[:] = 0.0
        q[q.size // 2] = 1.0e-3
        b.update()
        v = np.zeros(g.np, np.float32)
        v[g.np // 2] = 1.0e-3
        g.set("qext", v)
        g.step(1)
        assert np.array_equal(zs, g.get("zs").astype(np.float64))
        assert zs[q.size // 2] > before[q.size // 2]
    finally:
        g.close()
        b.finalize()
