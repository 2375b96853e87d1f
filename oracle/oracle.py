"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, as the checker; the shipped library never does.  See
``sfincs_oracle.cpp`` for what is restated and the parity status (unpinned
against reference outputs: the Fortran reference cannot be built here).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

SCALARS = ["t", "dt", "min_dt", "t0", "t1", "nt", "error", "dtmax", "dtmin", "np", "npuv",
           "nkcuv2", "ngbnd", "subgrid", "nlevels"]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
                os.path.join(_HERE, "sfincs_oracle.cpp")):
            build()
        L = ctypes.CDLL(_SO)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_update.restype = ctypes.c_long
        L.oracle_update.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_long]
        L.oracle_scalars.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.oracle_get.restype = ctypes.c_int
        L.oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_long]
        L.oracle_set.restype = ctypes.c_int
        L.oracle_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_long]
        _lib = L
    return _lib


class Oracle:
    """One oracle model instance read from ``<directory>/sfincs.inp``.

    precision: "fp64" (FP64-promoted), "ref" (the reference's mixed precision:
    zs and z_volume real*8, the rest real*4) or "f32" (the CUDA core's
    precision: zs float, z_volume double).
    """

    def __init__(self, directory: str, precision: str = "fp64", bmi: bool = False):
        L = lib()
        self._h = L.oracle_create(directory.encode(), precision.encode(), int(bmi))
        if not self._h:
            raise RuntimeError("oracle: " + L.oracle_last_error().decode())
        self.precision = precision

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def scalars(self) -> dict:
        buf = (ctypes.c_double * len(SCALARS))()
        lib().oracle_scalars(self._h, buf)
        return dict(zip(SCALARS, list(buf)))

    def update(self, dtrange: float = -1.0, max_steps: int = -1) -> int:
        """``sfincs_update(dtrange)``: -1 one step, >0 advance by dtrange, < -999 run to tstop."""
        return int(lib().oracle_update(self._h, float(dtrange), int(max_steps)))

    def run_to_end(self) -> int:
        return self.update(-1000.0)

    def update_until(self, t_target: float) -> int:
        return self.update(float(t_target) - self.scalars()["t"])

    def get(self, name: str, n: int | None = None) -> np.ndarray:
        """Copy a named array; n defaults to npuv for face arrays, nkcuv2 for
        uvmean and np otherwise (pass n for the boundary-face lists kb_*)."""
        if n is None:
            s = self.scalars()
            if name in ("q", "uv", "kfuv", "kcuv", "mask_adv", "uv_nm", "uv_nmu", "uv_dir"):
                n = int(s["npuv"])
            elif name == "uvmean":
                n = int(s["nkcuv2"])
            else:
                n = int(s["np"])
        out = np.zeros(n, np.float64)
        rc = lib().oracle_get(self._h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
        if rc != 0:
            raise KeyError(name)
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        rc = lib().oracle_set(self._h, name.encode(), v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), v.size)
        if rc != 0:
            raise KeyError(name)
