"""Input formats: sfincs.inp keyword rules, dates, netCDF-3 files, binary layout."""
import os

import numpy as np
import pytest

from sfincs_b200 import bmi as B
from sfincs_b200 import ncfile, synth


def test_netcdf3_roundtrip(tmp_path):
    p = str(tmp_path / "t.nc")
    a = np.arange(12, dtype=np.float32).reshape(4, 3)
    b = np.array([1, -2, 3], np.int32)
    c = np.linspace(0, 1, 5)
    ncfile.write(p, {"np": 4, "levels": 3, "k": 5}, {"a": (("np", "levels"), a), "b": (("levels",), b),
                                                     "c": (("k",), c)}, {"x0": 1.5, "name": "sbg"})
    dims, var, gat = ncfile.read(p)
    assert dims == {"np": 4, "levels": 3, "k": 5}
    assert np.array_equal(var["a"], a) and np.array_equal(var["b"], b) and np.allclose(var["c"], c)
    assert gat["name"] == "sbg" and float(gat["x0"][0]) == 1.5


def test_face_enumeration_reference_order():
    msk = np.ones((3, 4), np.int8)
    msk[0, 0] = 0
    f = synth.enumerate_faces(msk)
    # first active cell (n=1,m=0 0-based) owns a right face then an upper face
    assert f[0].tolist() == [0, 1, 0] and f[1].tolist() == [1, 1, 0]
    # every face joins two active cells
    for d, n, m in f:
        n2, m2 = (n, m + 1) if d == 0 else (n + 1, m)
        assert msk[n, m] > 0 and msk[n2, m2] > 0


def test_binary_files_follow_reference_layout(tmp_path):
    m = synth.plain_regular(nmax=5, mmax=6, dx=100.0, tstop=600.0, nbumps=1)
    m.msk[2, 3] = 0
    d = m.write(str(tmp_path))
    ind = np.fromfile(os.path.join(d, "sfincs.ind"), np.int32)
    assert ind[0] == (m.msk > 0).sum()
    idx = ind[1:]
    n = (idx - 1) % 5
    mm = (idx - 1) // 5
    assert np.all(m.msk[n, mm] > 0)
    assert np.all(np.diff(idx) > 0)  # n fastest, m outer: increasing linear index
    zb = np.fromfile(os.path.join(d, "sfincs.dep"), np.float32)
    assert np.allclose(zb, m.zb[n, mm])


def _write_inp(d, text):
    with open(os.path.join(d, "sfincs.inp"), "w", newline="") as f:
        f.write(text)


def test_inp_keyword_rules(tmp_path):
    """Comments, tabs, CR, trailing '#' comments, first occurrence wins
    (sfincs_read.f90:192-249); both the core and the oracle parse alike."""
    from oracle.oracle import Oracle

    m = synth.plain_regular(nmax=6, mmax=8, dx=200.0, tstop=600.0, nbumps=1)
    d = m.write(str(tmp_path))
    lines = open(os.path.join(d, "sfincs.inp")).read().splitlines()
    lines = [ln for ln in lines if not ln.startswith(("alpha", "tstart", "tstop", "tref", "huthresh"))]
    extra = [
        "# alpha = 0.9",
        "! a comment",
        "alpha\t= 0.35   # trailing comment",
        "alpha = 0.7",
        "hmin_cfl = 0.2\r",
        "tref = 20000101 000000",
        "tstart = 20000101 010000",
        "tstop = 20000102 000000",
        "huthresh = 0.02",
    ]
    _write_inp(d, "\n".join(lines + extra) + "\n")
    cnt = B.layout(d, "counts", 10)
    o = Oracle(d, "fp64")
    s = o.scalars()
    assert cnt[8] == 3600.0 and cnt[9] == 86400.0
    assert s["t0"] == 3600.0 and s["t1"] == 86400.0
    dtmax_expected = np.float32(min(60.0, np.float32(0.35) * np.float32(200.0) / np.sqrt(np.float32(9.81 * np.float32(0.2)))))
    assert cnt[6] == pytest.approx(float(dtmax_expected), rel=1e-6)
    assert cnt[6] == s["dtmax"]


def test_dates_across_month_and_leap_year(tmp_path):
    m = synth.plain_regular(nmax=4, mmax=5, dx=200.0, tstop=600.0, nbumps=1)
    m.params.update({"tref": "20000228 000000", "tstart": "20000228 120000", "tstop": "20000301 000000"})
    d = m.write(str(tmp_path))
    cnt = B.layout(d, "counts", 10)
    assert cnt[8] == 12 * 3600.0
    assert cnt[9] == 2 * 86400.0  # 2000 is a leap year: Feb 29 exists
