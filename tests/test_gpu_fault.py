"""The bounded wait of the staged (TMA) kernels, made to give up on purpose.

SFG_TEST_WAIT_ROUNDS=0 (read when a model is created) gives the mbarrier
wait for each tile's data no rounds at all: every tile is skipped, the
scenario's fault flag is set, the copies already issued are drained before
their stage is reused and before the CTA exits, and the run reports an error.
Nothing on the GPU faults: a model created afterwards on the same device runs
and matches the oracle."""
import os

import numpy as np
import pytest

from conftest import small_plain, small_subgrid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [small_plain, small_subgrid], ids=["plain", "subgrid"])
def test_wait_that_gives_up_sets_the_fault_and_the_context_survives(tmp_path, make):
    from oracle.oracle import Oracle
    from sfincs_b200.bmi import Model

    d, _ = make(tmp_path)
    os.environ["SFG_TEST_WAIT_ROUNDS"] = "0"
    try:
        g = Model(d)
    finally:
        del os.environ["SFG_TEST_WAIT_ROUNDS"]
    assert g.variant >= 4  # the staged (TMA) path
    with pytest.raises(RuntimeError, match="fault flag"):
        g.step(3)
    g.close()
    # the context still works: a fresh model steps and matches the oracle
    o = Oracle(d, "f32")
    g = Model(d)
    o.update(-1000.0, 20)
    g.step(20)
    assert float(np.abs(o.get("zs") - g.get("zs")).max()) <= 2e-5
    g.close()
