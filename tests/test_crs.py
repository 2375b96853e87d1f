"""Cross-sections (sfincs_crosssections.f90:8-176): the uv points each
polyline crosses, in uv-point order, and the sign of each crossing, on a
regular grid and a quadtree mesh, against the oracle face by face."""
import numpy as np
import pytest

from crs_cases import add_crs
from sfincs_b200 import bmi as B


def _faces(d, n_o):
    from oracle.oracle import Oracle

    o = Oracle(d, "f32")
    want = o.get("crs_faces", 4 * n_o).reshape(-1, 4)
    o.close()
    return want


@pytest.mark.parametrize("quadtree", [False, True])
def test_crossed_faces_and_signs_match_oracle(tmp_path, quadtree):
    from sfincs_b200 import qtsynth, synth

    if quadtree:
        m = qtsynth.quadtree_coastal(nmax1=8, mmax1=10, dx1=400.0, nlev=3, bands=(1000.0, 500.0), P=4, seed=21,
                                     tstop=1800.0, subgrid=False, wind_speed=0.0)
    else:
        m = synth.plain_regular(nmax=24, mmax=30, dx=400.0, tstop=1800.0, seed=3, nbumps=6)
    d = m.write(str(tmp_path))
    add_crs(d, scale=1.0 / 3.0 if quadtree else 1.0)  # the quadtree mesh spans 4 km x 3.2 km
    got = []
    for n in range(1, 400):  # the layout getter wants the exact length
        try:
            got = B.layout(d, "crs_faces", 4 * n).reshape(-1, 4)
            break
        except RuntimeError:
            continue
    assert len(got) > 20
    want = _faces(d, len(got))
    assert np.array_equal(got, want)
    for c in range(3):  # every polyline crosses faces, with both signs on the diagonal
        assert (got[:, 0] == c).sum() > 3
    diag = got[got[:, 0] == 2]
    assert set(diag[:, 2]) == {0.0, 1.0}


def test_crsfile_refused_on_geographic_grids(tmp_path):
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).parent))
    from geo_cases import geographic
    from sfincs_b200 import synth

    m = synth.plain_regular(nmax=12, mmax=14, dx=400.0, tstop=600.0, seed=3, nbumps=2)
    geographic(m)
    d = m.write(str(tmp_path))
    add_crs(d)
    with pytest.raises(RuntimeError, match="crsfile"):
        B.layout(d, "counts", 10)
