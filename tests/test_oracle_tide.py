"""Astronomic boundaries (bca files, sfincs_boundaries.f90:289-450, 736-744;
nodal factors of the vendored tidal package, Delft3D astro.f90).

The oracle's constituent speeds are checked against the published speeds, and
its nodal factors f and phase corrections u against the standard series in
the longitude of the moon's node N (Schureman's method, as tabulated in tidal
textbooks), with the equilibrium arguments V0 from the mean longitudes of the
moon, the sun and the lunar perigee (Meeus).  The core's host arrays equal the
oracle's bit for bit; the core's cosine is checked against float64 cos."""
import ctypes
import datetime as dt
import math
import os

import numpy as np
import pytest

from sfincs_b200 import bmi as B
from sfincs_b200 import synth
from tide_cases import MAIN, add_bca, set_tref


def _model(tmp_path, tref="20210315 060000", sets=None, extra=None, name="m"):
    m = synth.plain_regular(nmax=8, mmax=10, dx=400.0, tstop=600.0, seed=3, nbumps=1)
    d = m.write(str(tmp_path / name))
    set_tref(d, tref)
    add_bca(d, sets if sets is not None else [[(c, 1.0, 0.0) for c in MAIN]], extra)
    return d


def _oracle(d):
    from oracle.oracle import Oracle

    return Oracle(d, "f32")


# Published constituent speeds, degrees per mean solar hour.
SPEEDS = {"M2": 28.9841042, "S2": 30.0, "N2": 28.4397295, "K2": 30.0821373, "K1": 15.0410686, "O1": 13.9430356,
          "P1": 14.9589314, "Q1": 13.3986609, "MF": 1.0980331, "MM": 0.5443747, "M4": 57.9682084,
          "MS4": 58.9841042, "MN4": 57.4238337}


def test_constituent_speeds_are_the_published_ones(tmp_path):
    d = _model(tmp_path)
    nc = len(MAIN) + 1
    w = _oracle(d).get("tide_omega", nc)
    assert w[0] == 0.0  # A0
    for k, c in enumerate(MAIN):
        assert math.degrees(w[k + 1]) * 3600.0 == pytest.approx(SPEEDS[c], abs=2e-7), c


def _mean_longitudes(tref):
    """Hour angle of the mean sun + 180 deg, s, h, p and N (degrees) at tref,
    from the mean elements of Meeus (Astronomical Algorithms, ch. 47 / 22)."""
    d = dt.datetime.strptime(tref, "%Y%m%d %H%M%S")
    T = (d - dt.datetime(2000, 1, 1, 12)).total_seconds() / 86400.0 / 36525.0
    s = 218.3164477 + 481267.88123421 * T
    h = 280.46646 + 36000.76983 * T
    p = 83.3532465 + 4069.0137287 * T
    N = 125.04452 - 1934.136261 * T
    tau = 180.0 + 15.0 * (d.hour + d.minute / 60.0 + d.second / 3600.0)
    return tau, s, h, p, N


@pytest.mark.parametrize("year", [2000, 2004, 2009, 2013, 2018, 2022, 2026])
def test_nodal_factors_follow_the_standard_series(tmp_path, year):
    """f and u of M2, N2, S2, K1, O1 and K2 over a nodal cycle against
    f(N), u(N) series (M2: 1.0004 - 0.0373 cos N + 0.0002 cos 2N, -2.14 sin N;
    K1: 1.0060 + 0.1150 cos N - 0.0088 cos 2N + 0.0006 cos 3N, -8.86 sin N +
    0.68 sin 2N - 0.07 sin 3N; O1: 1.0089 + 0.1871 cos N - 0.0147 cos 2N +
    0.0014 cos 3N, 10.80 sin N - 1.34 sin 2N + 0.19 sin 3N; K2: 1.0241 +
    0.2863 cos N + 0.0083 cos 2N - 0.0015 cos 3N, -17.74 sin N + 0.68 sin 2N -
    0.04 sin 3N)."""
    tref = f"{year}0315 060000"
    d = _model(tmp_path, tref)
    o = _oracle(d)
    nc = len(MAIN) + 1
    A, P = o.get("tide_amp", nc), o.get("tide_phase", nc)
    tau, s, h, p, N = _mean_longitudes(tref)
    n = math.radians(N)
    c1, c2, c3 = math.cos(n), math.cos(2 * n), math.cos(3 * n)
    s1, s2, s3 = math.sin(n), math.sin(2 * n), math.sin(3 * n)
    fm2, um2 = 1.0004 - 0.0373 * c1 + 0.0002 * c2, -2.14 * s1
    want = {
        "M2": (2 * tau - 2 * s + 2 * h, fm2, um2),
        "N2": (2 * tau - 3 * s + 2 * h + p, fm2, um2),
        "S2": (2 * tau, 1.0, 0.0),
        "K1": (tau + h - 90.0, 1.0060 + 0.1150 * c1 - 0.0088 * c2 + 0.0006 * c3, -8.86 * s1 + 0.68 * s2 - 0.07 * s3),
        "O1": (tau - 2 * s + h + 90.0, 1.0089 + 0.1871 * c1 - 0.0147 * c2 + 0.0014 * c3,
               10.80 * s1 - 1.34 * s2 + 0.19 * s3),
        "K2": (2 * tau + 2 * h, 1.0241 + 0.2863 * c1 + 0.0083 * c2 - 0.0015 * c3, -17.74 * s1 + 0.68 * s2 - 0.04 * s3),
    }
    for c, (v0, f, u) in want.items():
        i = MAIN.index(c) + 1
        v0u = math.degrees(-P[i]) % 360.0  # the phase of a 0-degree input is -(V0 + u) mod 2 pi
        got_u = (v0u - v0 + 180.0) % 360.0 - 180.0
        assert A[i] == pytest.approx(f, abs=2e-3), (c, A[i], f)
        assert got_u == pytest.approx(u, abs=0.12), (c, got_u, u)
        assert 0.0 <= P[i] < 2 * math.pi + 1e-12


@pytest.mark.parametrize("tref", ["20210315 060000", "20160229 235959", "19951231 123456", "20240101 000000"])
def test_core_arrays_equal_the_oracle(tmp_path, tref):
    """Two points, different amplitudes and phases, the first set led by A0, a
    renamed constituent (EPS2): the core's host arrays are the oracle's."""
    rng = np.random.default_rng(3)
    comps = ["A0", "M2", "S2", "EPS2", "K1", "O1", "MF", "M4", "LA2", "MTM", "SA"]
    sets = [[(c, float(rng.uniform(0.01, 1.2)), float(rng.uniform(-360, 720))) for c in comps] for _ in range(2)]
    m = synth.plain_regular(nmax=8, mmax=10, dx=400.0, tstop=600.0, seed=3, nbumps=1)
    m.bnd = np.array([[0.0, 400.0], [0.0, 2800.0]])
    m.bzs = np.stack([m.bzs[:, 0], m.bzs[:, 1], 0.5 * m.bzs[:, 1]], axis=1)
    d = m.write(str(tmp_path / "two"))
    set_tref(d, tref)
    add_bca(d, sets)
    o = _oracle(d)
    nc = len(comps)
    for name, n in (("tide_omega", nc), ("tide_amp", 2 * nc), ("tide_phase", 2 * nc)):
        a, b = B.layout(d, name, n), o.get(name, n)
        assert np.array_equal(a, b), name
    amp = B.layout(d, "tide_amp", 2 * nc)
    written = [np.float32(f"{sets[k][0][1]:.5f}") for k in range(2)]  # as the bca file holds them
    assert amp[0] == written[0] and amp[nc] == written[1]  # A0: no nodal factor
    assert B.layout(d, "tide_omega", nc)[0] == 0.0


def test_without_a0_the_first_constituent_is_a_zero_a0(tmp_path):
    d = _model(tmp_path, sets=[[("M2", 0.8, 30.0), ("S2", 0.3, 60.0)]])
    w, a = B.layout(d, "tide_omega", 3), B.layout(d, "tide_amp", 3)
    assert w[0] == 0.0 and a[0] == 0.0 and a[1] > 0.7
    assert np.array_equal(a, _oracle(d).get("tide_amp", 3))


def test_use_bcafile_off_ignores_the_file(tmp_path):
    d = _model(tmp_path, extra={"use_bcafile": 0})
    assert B.layout(d, "tide_omega", 0).size == 0


@pytest.mark.parametrize("case", ["unknown", "sets", "longer"])
def test_bca_refusals(tmp_path, case):
    if case == "unknown":
        sets = [[("M2", 1.0, 0.0), ("XX7", 0.1, 0.0)]]
    elif case == "sets":
        sets = [[("M2", 1.0, 0.0)], [("M2", 1.0, 0.0)]]  # two blocks, one boundary point
    else:
        sets = None
    d = _model(tmp_path, sets=sets)
    if case == "longer":  # a second block longer than the first needs a second point
        m = synth.plain_regular(nmax=8, mmax=10, dx=400.0, tstop=600.0, seed=3, nbumps=1)
        m.bnd = np.array([[0.0, 400.0], [0.0, 2800.0]])
        m.bzs = np.stack([m.bzs[:, 0], m.bzs[:, 1], m.bzs[:, 1]], axis=1)
        d = m.write(str(tmp_path / "longer"))
        add_bca(d, [[("M2", 1.0, 0.0)], [("M2", 1.0, 0.0), ("S2", 1.0, 0.0)]])
    with pytest.raises(RuntimeError):
        B.layout(d, "counts", 10)


def test_core_cosine_is_within_an_ulp_of_float64_cos():
    from oracle.oracle import lib

    f = lib().oracle_core_cos
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double]
    rng = np.random.default_rng(11)
    xs = np.concatenate([rng.uniform(-7.0, 7.0, 3000), rng.uniform(-2.0e4, 2.0e4, 3000),
                         np.arange(-40, 41) * (math.pi / 4), [0.0, 1e-300, 5e-324]])
    worst = 0.0
    for x in xs:
        got, want = f(float(x)), math.cos(float(x))
        ulps = abs(got - want) / float(np.spacing(abs(want)))
        worst = max(worst, ulps)
        assert ulps <= 3.0 or abs(got - want) <= 1e-19, (x, got, want)
    assert worst <= 3.0, worst
