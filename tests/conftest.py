import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (checker) and the CUDA library once per session."""
    from oracle import oracle
    from sfincs_b200 import build

    oracle.build()
    build.build()


def small_plain(tmpdir, nmax=24, mmax=30, dx=400.0, tstop=1800.0, seed=3, **params):
    from sfincs_b200 import synth

    m = synth.plain_regular(nmax=nmax, mmax=mmax, dx=dx, tstop=tstop, seed=seed, nbumps=6)
    m.params.update(params)
    return m.write(str(tmpdir)), m


def small_subgrid(tmpdir, nmax=20, mmax=24, dx=500.0, P=8, tstop=3600.0, seed=5, rain=40.0, **params):
    from sfincs_b200 import synth

    m = synth.subgrid_regular(nmax=nmax, mmax=mmax, dx=dx, P=P, seed=seed, tstop=tstop, rain_mmh=rain,
                              rain_hours=0.5, coast_x=mmax * dx * 0.3, t_peak=tstop / 2, width_h=0.5,
                              surge_peak=1.5)
    m.params.update(params)
    return m.write(str(tmpdir)), m


def oracle_faces_to_cells(o, arr):
    """Map an oracle per-face array (reference ip order) to (x, y) per-cell arrays
    in compact cell order: x = each cell's right (u) face, y = its upper (v) face."""
    s = o.scalars()
    n = int(s["np"])
    nm = o.get("uv_nm").astype(np.int64) - 1
    d = o.get("uv_dir").astype(np.int64)
    x = np.zeros(n)
    y = np.zeros(n)
    x[nm[d == 0]] = arr[d == 0]
    y[nm[d == 1]] = arr[d == 1]
    return x, y
