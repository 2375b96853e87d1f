"""Batched ensembles: members of different sizes and end times advanced by the
same launches give bitwise the states each member reaches alone."""
import numpy as np
import pytest

from sfincs_b200.bmi import Ensemble, Model

pytestmark = pytest.mark.gpu


def _members(tmp_path):
    from sfincs_b200 import synth

    dirs = []
    for i, (n, m, tstop, peak, rain) in enumerate([(16, 20, 1800.0, 1.0, 60.0), (24, 30, 2400.0, 2.5, 0.0),
                                                   (40, 28, 1200.0, 3.5, 20.0)]):
        d = tmp_path / f"m{i}"
        d.mkdir()
        mdl = synth.subgrid_regular(nmax=n, mmax=m, dx=400.0, P=6, seed=11 + i, tstop=tstop, surge_peak=peak,
                                    rain_mmh=rain, rain_hours=0.25, coast_x=m * 400.0 * 0.3, t_peak=tstop / 2,
                                    width_h=0.3)
        dirs.append(mdl.write(str(d)))
    return dirs


@pytest.mark.parametrize("autotune", [False, True])
def test_members_alone_equal_members_in_mix(tmp_path, autotune):
    dirs = _members(tmp_path)
    e = Ensemble(dirs)
    if autotune:
        e.set_autotune(True)
    t1 = [e.scalars(i)["t1"] for i in range(len(dirs))]
    e.run(t1)
    dts = set()
    for i, d in enumerate(dirs):
        g = Model(d)
        g.run(g.scalars()["t1"])
        se, sg = e.scalars(i), g.scalars()
        assert se["nt"] == sg["nt"] and se["t"] == sg["t"], (i, se["nt"], sg["nt"])
        assert se["t"] >= t1[i]
        dts.add(sg["dt"])
        for name in ("zs", "qx", "qy", "uvx", "uvy", "zsmax", "z_volume"):
            assert np.array_equal(e.get(i, name), g.get(name)), (i, name)
        g.close()
    assert len(dts) > 1  # members really step with their own dt
    if autotune:
        assert e.variant in (2, 4, 5)
    e.close()
