"""The allocation-free volume entry point agrees with the allocating one.

sfg_model_volume_noalloc keeps its scratch in a fixed array inside the
library; this file is collected last so it also runs after every other GPU
test has used the device."""
import pytest
from conftest import small_plain, small_subgrid

from sfincs_b200.bmi import Model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["plain", "subgrid"])
def test_noalloc_volume_matches_allocating_entry_point(tmp_path, kind):
    d, _ = (small_plain if kind == "plain" else small_subgrid)(tmp_path)
    m = Model(d)
    try:
        for nsteps in (0, 25, 40):
            if nsteps:
                m.step(nsteps)
            ref = m.volume()
            a = m.volume_noalloc()
            b = m.volume_noalloc()  # second call in a row reuses the scratch
            assert a == ref and b == ref, (kind, nsteps, ref, a, b)
            assert m.volume() == ref
    finally:
        m.close()


def test_noalloc_volume_two_models_in_turn(tmp_path):
    """Two models on the same device share the scratch array; calls made one
    after the other (never overlapping) each get their own model's sum."""
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    a, b = Model(small_plain(tmp_path / "a")[0]), Model(small_subgrid(tmp_path / "b")[0])
    try:
        a.step(10)
        b.step(10)
        va, vb = a.volume(), b.volume()
        for _ in range(2):
            assert a.volume_noalloc() == va
            assert b.volume_noalloc() == vb
    finally:
        a.close()
        b.close()
