"""ctypes binding of libsfincs_gpu.so.

``BMI`` drives the library exactly like xmipy drives the reference's
``libsfincs`` (``sfincs_bmi.f90``): one global model per process, by-reference
arguments, host pointers from ``get_value_ptr``.  ``Model`` and ``Ensemble``
wrap the handle APIs (independent models; uneven ensembles advanced by the same
launches).

The library is the only compute path: if it cannot be loaded the import fails
loudly (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libsfincs_gpu.so")
_lib = None

SCALARS = ["t", "dt", "min_dt", "nt", "error", "t0", "t1", "np", "npuv", "nkcuv2", "ngbnd", "subgrid",
           "bflux_vol", "rain_vol", "src_vol", "dtmax", "dtmin", "device_bytes", "ntiles"]

BMI_FUNCTIONS = ["initialize", "update", "update_until", "finalize", "get_value_ptr", "get_var_shape",
                 "get_var_type", "get_var_rank", "set_logical", "get_start_time", "get_end_time",
                 "get_time_step", "get_current_time", "update_zbuv", "update_apparent_roughness",
                 "get_sfincs_cell_index", "get_sfincs_cell_indices", "get_sfincs_cell_area",
                 "get_last_bmi_error"]
BMI_CONSTANTS = ["BMI_LENVARADDRESS", "BMI_LENVARTYPE", "BMI_LENGRIDTYPE", "BMI_LENCOMPONENTNAME",
                 "BMI_LENVERSION", "BMI_LENERRMESSAGE"]


def lib(build_if_missing: bool = True):
    """Load libsfincs_gpu.so (building it in-tree if it is missing here)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise RuntimeError(f"libsfincs_gpu.so not built ({LIB_PATH}); run sfincs_b200/build.py")
        from . import build as _b

        _b.build()
    L = ctypes.CDLL(LIB_PATH)
    c_dp = ctypes.POINTER(ctypes.c_double)
    c_ip = ctypes.POINTER(ctypes.c_int)
    L.initialize.restype = ctypes.c_int
    L.initialize_config.argtypes = [ctypes.c_char_p]
    L.update_until.argtypes = [ctypes.c_double]
    L.get_value_ptr.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]
    L.get_var_shape.argtypes = [ctypes.c_char_p, c_ip]
    L.get_var_type.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    L.get_var_rank.argtypes = [ctypes.c_char_p, c_ip]
    L.set_logical.argtypes = [ctypes.c_char_p, c_ip]
    for f in ("get_start_time", "get_end_time", "get_time_step", "get_current_time"):
        getattr(L, f).argtypes = [c_dp]
    L.get_sfincs_cell_index.argtypes = [c_dp, c_dp, c_ip]
    L.get_sfincs_cell_indices.argtypes = [c_dp, c_dp, c_ip, ctypes.c_int]
    L.get_sfincs_cell_area.argtypes = [c_ip, c_dp]
    L.get_last_bmi_error.argtypes = [ctypes.c_char_p]
    L.get_var.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.set_var.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.sfg_model_create.restype = ctypes.c_void_p
    L.sfg_model_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.sfg_model_destroy.argtypes = [ctypes.c_void_p]
    L.sfg_model_finalize.argtypes = [ctypes.c_void_p]
    L.sfg_model_run.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_longlong, ctypes.c_int]
    L.sfg_model_issue.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.sfg_model_sync.argtypes = [ctypes.c_void_p]
    L.sfg_model_scalars.argtypes = [ctypes.c_void_p, c_dp]
    L.sfg_model_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.sfg_model_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.sfg_model_volume.argtypes = [ctypes.c_void_p, c_dp]
    for f in ("sfg_model_set_autotune", "sfg_model_set_variant", "sfg_ensemble_set_autotune",
              "sfg_ensemble_set_variant"):
        getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
    for f in ("sfg_model_variant", "sfg_ensemble_variant"):
        getattr(L, f).argtypes = [ctypes.c_void_p]
    L.sfg_model_volume_noalloc.argtypes = [ctypes.c_void_p, c_dp]
    L.sfg_model_stream.restype = ctypes.c_void_p
    L.sfg_model_stream.argtypes = [ctypes.c_void_p]
    L.sfg_ensemble_create.restype = ctypes.c_void_p
    L.sfg_ensemble_create.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int,
                                      ctypes.c_char_p, ctypes.c_int]
    L.sfg_ensemble_destroy.argtypes = [ctypes.c_void_p]
    L.sfg_ensemble_run.argtypes = [ctypes.c_void_p, c_dp, ctypes.c_longlong, ctypes.c_int]
    L.sfg_ensemble_issue.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.sfg_ensemble_sync.argtypes = [ctypes.c_void_p]
    L.sfg_ensemble_scalars.argtypes = [ctypes.c_void_p, ctypes.c_int, c_dp]
    L.sfg_ensemble_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.sfg_ensemble_stream.restype = ctypes.c_void_p
    L.sfg_ensemble_stream.argtypes = [ctypes.c_void_p]
    L.sfg_model_kernel_times.argtypes = [ctypes.c_void_p, ctypes.c_int, c_dp, c_ip]
    L.sfg_ensemble_kernel_times.argtypes = [ctypes.c_void_p, ctypes.c_int, c_dp, c_ip]
    L.sfg_layout_get.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, c_dp, ctypes.c_size_t]
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().get_last_bmi_error(buf)
    return buf.value.decode()


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed ({rc}): {last_error()}")


_F32_NAMES = {"zsmax", "qext", "qx", "qy", "uvx", "uvy", "zs0", "zsderv", "vmax", "qmax", "twet", "tzsmax", "cumprcp", "cuminf"}
_F64_NAMES = {"zs", "z_volume"}


def _alloc(name: str, n: int) -> np.ndarray:
    if name in _F64_NAMES:
        return np.zeros(n, np.float64)
    if name == "kfuv":
        return np.zeros(2 * n, np.float32)
    return np.zeros(n, np.float32)


def layout(model_dir: str, name: str, n: int, bmi: bool = False) -> np.ndarray:
    """Host-side layout array of a model (no device work); see sfg_layout_get."""
    out = np.zeros(n, np.float64)
    _check(lib().sfg_layout_get(model_dir.encode(), int(bmi), name.encode(),
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n), f"layout({name})")
    return out


class BMI:
    """The reference's BMI surface (``sfincs_bmi.f90``), one model per process."""

    def __init__(self):
        self.L = lib()

    def initialize(self, model_dir: str | None = None) -> None:
        rc = self.L.initialize() if model_dir is None else self.L.initialize_config(model_dir.encode())
        _check(rc, "initialize")

    def update(self) -> None:
        _check(self.L.update(), "update")

    def update_until(self, t: float) -> None:
        _check(self.L.update_until(float(t)), "update_until")

    def finalize(self) -> int:
        return int(self.L.finalize())

    def get_value_ptr(self, name: str) -> np.ndarray:
        p = ctypes.c_void_p()
        _check(self.L.get_value_ptr(name.encode(), ctypes.byref(p)), f"get_value_ptr({name})")
        shape = (ctypes.c_int * 6)()
        _check(self.L.get_var_shape(name.encode(), shape), "get_var_shape")
        t = ctypes.create_string_buffer(64)
        _check(self.L.get_var_type(name.encode(), t), "get_var_type")
        ct = {"float": ctypes.c_float, "double": ctypes.c_double, "integer": ctypes.c_int}[t.value.decode()]
        arr = ctypes.cast(p, ctypes.POINTER(ct * shape[0])).contents
        return np.ctypeslib.as_array(arr)

    def get_var_type(self, name: str) -> str:
        t = ctypes.create_string_buffer(64)
        _check(self.L.get_var_type(name.encode(), t), "get_var_type")
        return t.value.decode()

    def get_var_rank(self, name: str) -> int:
        r = ctypes.c_int()
        _check(self.L.get_var_rank(name.encode(), ctypes.byref(r)), "get_var_rank")
        return r.value

    def get_var_shape(self, name: str) -> tuple:
        s = (ctypes.c_int * 6)()
        _check(self.L.get_var_shape(name.encode(), s), "get_var_shape")
        return tuple(x for x in s if x)

    def set_logical(self, name: str, value: bool) -> None:
        v = ctypes.c_int(1 if value else 0)
        _check(self.L.set_logical(name.encode(), ctypes.byref(v)), "set_logical")

    def _time(self, fn) -> float:
        x = ctypes.c_double()
        _check(getattr(self.L, fn)(ctypes.byref(x)), fn)
        return x.value

    def get_start_time(self) -> float:
        return self._time("get_start_time")

    def get_end_time(self) -> float:
        return self._time("get_end_time")

    def get_time_step(self) -> float:
        return self._time("get_time_step")

    def get_current_time(self) -> float:
        return self._time("get_current_time")

    def update_zbuv(self) -> None:
        _check(self.L.update_zbuv(), "update_zbuv")

    def get_sfincs_cell_index(self, x: float, y: float) -> int:
        i = ctypes.c_int()
        _check(self.L.get_sfincs_cell_index(ctypes.byref(ctypes.c_double(x)), ctypes.byref(ctypes.c_double(y)),
                                            ctypes.byref(i)), "get_sfincs_cell_index")
        return i.value

    def get_sfincs_cell_indices(self, x, y) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        out = np.zeros(x.size, np.int32)
        c_dp = ctypes.POINTER(ctypes.c_double)
        _check(self.L.get_sfincs_cell_indices(x.ctypes.data_as(c_dp), y.ctypes.data_as(c_dp),
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), x.size),
               "get_sfincs_cell_indices")
        return out

    def get_sfincs_cell_area(self, index: int) -> float:
        a = ctypes.c_double()
        _check(self.L.get_sfincs_cell_area(ctypes.byref(ctypes.c_int(index)), ctypes.byref(a)), "get_sfincs_cell_area")
        return a.value

    def get_var(self, name: str, n: int) -> np.ndarray:
        out = _alloc(name, n)
        _check(self.L.get_var(name.encode(), out.ctypes.data, out.nbytes), f"get_var({name})")
        return out

    def set_var(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, np.float64 if name in _F64_NAMES else np.float32)
        _check(self.L.set_var(name.encode(), v.ctypes.data, v.nbytes), f"set_var({name})")


class Model:
    """An independent device-resident model (handle API)."""

    def __init__(self, model_dir: str, bmi: bool = False):
        self.L = lib()
        err = ctypes.create_string_buffer(1024)
        self._h = self.L.sfg_model_create(model_dir.encode(), int(bmi), err, 1024)
        if not self._h:
            raise RuntimeError("sfg_model_create: " + err.value.decode())
        self.np = int(self.scalars()["np"])

    def finalize(self):
        """finalize_output: the last max interval, the run's scalars, the output files closed."""
        _check(self.L.sfg_model_finalize(self._h), "sfg_model_finalize")

    def close(self):
        if getattr(self, "_h", None):
            self.L.sfg_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, t_end: float, max_steps: int = -1, chunk: int = 32) -> None:
        _check(self.L.sfg_model_run(self._h, float(t_end), int(max_steps), int(chunk)), "sfg_model_run")

    def step(self, n: int = 1) -> None:
        """Exactly n steps (bounded by tstop like the reference's loop)."""
        s = self.scalars()
        self.run(s["t1"], max_steps=n, chunk=max(1, min(n, 32)))

    def issue(self, nsteps: int) -> None:
        _check(self.L.sfg_model_issue(self._h, int(nsteps)), "sfg_model_issue")

    def sync(self) -> None:
        _check(self.L.sfg_model_sync(self._h), "sfg_model_sync")

    def scalars(self) -> Dict[str, float]:
        buf = (ctypes.c_double * 19)()
        _check(self.L.sfg_model_scalars(self._h, buf), "sfg_model_scalars")
        return dict(zip(SCALARS, list(buf)))

    def get(self, name: str) -> np.ndarray:
        out = _alloc(name, self.np)
        _check(self.L.sfg_model_get(self._h, name.encode(), out.ctypes.data, out.nbytes), f"get({name})")
        return out

    def set(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, np.float64 if name in _F64_NAMES else np.float32)
        _check(self.L.sfg_model_set(self._h, name.encode(), v.ctypes.data, v.nbytes), f"set({name})")

    def volume(self) -> float:
        v = ctypes.c_double()
        _check(self.L.sfg_model_volume(self._h, ctypes.byref(v)), "sfg_model_volume")
        return v.value

    @property
    def variant(self) -> int:
        return int(self.L.sfg_model_variant(self._h))

    def set_variant(self, v: int) -> None:
        _check(self.L.sfg_model_set_variant(self._h, int(v)), "sfg_model_set_variant")

    def set_autotune(self, on: bool = True) -> None:
        _check(self.L.sfg_model_set_autotune(self._h, int(bool(on))), "sfg_model_set_autotune")

    def volume_noalloc(self) -> float:
        """volume() through the entry point that allocates nothing (fixed
        scratch array in the library, shared per device: do not overlap calls)."""
        v = ctypes.c_double()
        _check(self.L.sfg_model_volume_noalloc(self._h, ctypes.byref(v)), "sfg_model_volume_noalloc")
        return v.value

    @property
    def stream(self) -> int:
        return int(self.L.sfg_model_stream(self._h) or 0)

    def kernel_times(self, nsteps: int):
        """Mean ms per launch of [step+boundary, momentum, sources, continuity] and launches per step."""
        out = (ctypes.c_double * 4)()
        lps = ctypes.c_int()
        _check(self.L.sfg_model_kernel_times(self._h, int(nsteps), out, ctypes.byref(lps)), "kernel_times")
        return list(out), lps.value


class Ensemble:
    """Many uneven models advanced together by the same launches (per-member dt)."""

    def __init__(self, model_dirs: Sequence[str], bmi: bool = False):
        self.L = lib()
        arr = (ctypes.c_char_p * len(model_dirs))(*[d.encode() for d in model_dirs])
        err = ctypes.create_string_buffer(1024)
        self._h = self.L.sfg_ensemble_create(arr, len(model_dirs), int(bmi), err, 1024)
        if not self._h:
            raise RuntimeError("sfg_ensemble_create: " + err.value.decode())
        self.n = len(model_dirs)
        self.nps = [int(self.scalars(i)["np"]) for i in range(self.n)]

    def close(self):
        if getattr(self, "_h", None):
            self.L.sfg_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, t_end: Sequence[float], max_steps: int = -1, chunk: int = 32) -> None:
        te = np.ascontiguousarray(t_end, np.float64)
        _check(self.L.sfg_ensemble_run(self._h, te.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(max_steps),
                                       int(chunk)), "sfg_ensemble_run")

    def issue(self, nsteps: int) -> None:
        _check(self.L.sfg_ensemble_issue(self._h, int(nsteps)), "sfg_ensemble_issue")

    @property
    def variant(self) -> int:
        return int(self.L.sfg_ensemble_variant(self._h))

    def set_variant(self, v: int) -> None:
        _check(self.L.sfg_ensemble_set_variant(self._h, int(v)), "sfg_ensemble_set_variant")

    def set_autotune(self, on: bool = True) -> None:
        _check(self.L.sfg_ensemble_set_autotune(self._h, int(bool(on))), "sfg_ensemble_set_autotune")

    def sync(self) -> None:
        _check(self.L.sfg_ensemble_sync(self._h), "sfg_ensemble_sync")

    def scalars(self, i: int) -> Dict[str, float]:
        buf = (ctypes.c_double * 19)()
        _check(self.L.sfg_ensemble_scalars(self._h, i, buf), "sfg_ensemble_scalars")
        return dict(zip(SCALARS, list(buf)))

    def get(self, i: int, name: str) -> np.ndarray:
        out = _alloc(name, self.nps[i])
        _check(self.L.sfg_ensemble_get(self._h, i, name.encode(), out.ctypes.data, out.nbytes), f"get({name})")
        return out

    @property
    def stream(self) -> int:
        return int(self.L.sfg_ensemble_stream(self._h) or 0)

    def kernel_times(self, nsteps: int):
        out = (ctypes.c_double * 4)()
        lps = ctypes.c_int()
        _check(self.L.sfg_ensemble_kernel_times(self._h, int(nsteps), out, ctypes.byref(lps)), "kernel_times")
        return list(out), lps.value
