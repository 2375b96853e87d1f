"""Serving loop: continuous batching of forecast/ensemble requests on one GPU.

Requests arrive over time (model directory + end time).  Each one is prepared
on a host thread as soon as it arrives (input files -> dense layout, no device
work), admitted into the device pool when a slot is free and its exact device
footprint fits the HBM budget, advanced together with every other resident
request in the same launches, and retired as soon as it reaches its end time
(results copied out, memory released).  Requests that arrive while others
are running join at the next chunk boundary, so their work overlaps on the
device.  ``Server.serve`` returns per-request latency (arrival -> results on
the host) and the run's throughput.
"""
from __future__ import annotations

import ctypes
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from .bmi import SCALARS, _alloc, _check, lib


def _bind(L):
    if getattr(L, "_pool_bound", False):
        return L
    c_dp = ctypes.POINTER(ctypes.c_double)
    L.sfg_pool_create.restype = ctypes.c_void_p
    L.sfg_pool_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_int]
    L.sfg_pool_destroy.argtypes = [ctypes.c_void_p]
    L.sfg_prepare.restype = ctypes.c_void_p
    L.sfg_prepare.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.sfg_prepared_bytes.restype = ctypes.c_double
    L.sfg_prepared_bytes.argtypes = [ctypes.c_void_p]
    L.sfg_prepared_cells.restype = ctypes.c_double
    L.sfg_prepared_cells.argtypes = [ctypes.c_void_p]
    L.sfg_prepared_destroy.argtypes = [ctypes.c_void_p]
    L.sfg_pool_admit.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    L.sfg_pool_advance.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.sfg_pool_finished.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    L.sfg_pool_scalars.argtypes = [ctypes.c_void_p, ctypes.c_int, c_dp]
    L.sfg_pool_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t]
    L.sfg_pool_release.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.sfg_pool_used_bytes.restype = ctypes.c_double
    L.sfg_pool_used_bytes.argtypes = [ctypes.c_void_p]
    L.sfg_pool_resident.argtypes = [ctypes.c_void_p]
    L.sfg_pool_stream.restype = ctypes.c_void_p
    L.sfg_pool_stream.argtypes = [ctypes.c_void_p]
    L._pool_bound = True
    return L


class Prepared:
    """A model read and laid out on the host, not yet on the device."""

    def __init__(self, model_dir: str, bmi: bool = False):
        self.L = _bind(lib())
        err = ctypes.create_string_buffer(1024)
        self._h = self.L.sfg_prepare(model_dir.encode(), int(bmi), err, 1024)
        if not self._h:
            raise RuntimeError("sfg_prepare: " + err.value.decode())
        self.bytes = int(self.L.sfg_prepared_bytes(self._h))
        self.cells = int(self.L.sfg_prepared_cells(self._h))

    def release(self):
        if self._h:
            self.L.sfg_prepared_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Pool:
    """Device pool of resident models (C-ABI ``sfg_pool_*``)."""

    def __init__(self, max_slots: int, hbm_budget_bytes: float):
        self.L = _bind(lib())
        err = ctypes.create_string_buffer(1024)
        self._h = self.L.sfg_pool_create(int(max_slots), float(hbm_budget_bytes), err, 1024)
        if not self._h:
            raise RuntimeError("sfg_pool_create: " + err.value.decode())
        self.max_slots = max_slots
        self.nps: Dict[int, int] = {}

    def close(self):
        if getattr(self, "_h", None):
            self.L.sfg_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, prep: Prepared, t_end: float) -> int:
        k = self.L.sfg_pool_admit(self._h, prep._h, float(t_end))
        if k == -2:
            _check(-1, "sfg_pool_admit")
        if k >= 0:
            prep._h = None  # consumed by the pool
            self.nps[k] = prep.cells
        return k

    def advance(self, nsteps: int) -> int:
        r = self.L.sfg_pool_advance(self._h, int(nsteps))
        if r < 0:
            _check(-1, "sfg_pool_advance")
        return r

    def finished(self) -> List[int]:
        buf = (ctypes.c_int * self.max_slots)()
        c = self.L.sfg_pool_finished(self._h, buf, self.max_slots)
        return [buf[i] for i in range(c)]

    def scalars(self, slot: int) -> Dict[str, float]:
        buf = (ctypes.c_double * 19)()
        _check(self.L.sfg_pool_scalars(self._h, slot, buf), "sfg_pool_scalars")
        return dict(zip(SCALARS, list(buf)))

    def get(self, slot: int, name: str) -> np.ndarray:
        out = _alloc(name, self.nps[slot])
        _check(self.L.sfg_pool_get(self._h, slot, name.encode(), out.ctypes.data, out.nbytes), f"pool get({name})")
        return out

    def release(self, slot: int) -> None:
        _check(self.L.sfg_pool_release(self._h, slot), "sfg_pool_release")
        self.nps.pop(slot, None)

    @property
    def used_bytes(self) -> int:
        return int(self.L.sfg_pool_used_bytes(self._h))

    @property
    def resident(self) -> int:
        return int(self.L.sfg_pool_resident(self._h))


@dataclass
class Request:
    arrival_s: float          # seconds after serve() starts
    model_dir: str
    t_end: Optional[float] = None  # default: the model's own tstop
    rid: int = 0


@dataclass
class Result:
    rid: int
    arrival_s: float
    admitted_s: float
    done_s: float
    cells: int
    steps: int
    sim_t: float
    error: int
    fields: Dict[str, np.ndarray] = field(default_factory=dict)

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


class Server:
    """Continuous-batching request loop over a ``Pool``.

    max_slots: resident requests at most; hbm_budget_bytes: device bytes the
    resident requests may hold together; chunk: steps per advance (the
    admission/retirement granularity); prep_threads: host threads preparing
    arrived requests."""

    def __init__(self, max_slots: int = 32, hbm_budget_bytes: Optional[float] = None, chunk: int = 32,
                 prep_threads: int = 4):
        if hbm_budget_bytes is None:
            import torch

            free, _ = torch.cuda.mem_get_info()
            hbm_budget_bytes = 0.7 * free
        self.pool = Pool(max_slots, hbm_budget_bytes)
        self.budget = hbm_budget_bytes
        self.chunk = chunk
        self.prep_threads = prep_threads

    def close(self):
        self.pool.close()

    def serve(self, requests: Sequence[Request], fetch: Sequence[str] = ("zs",)) -> Dict:
        reqs = sorted(requests, key=lambda r: r.arrival_s)
        results: List[Result] = []
        ex = ThreadPoolExecutor(max_workers=self.prep_threads)
        futures = []          # (request, future) in arrival order
        ready: List = []      # (request, Prepared) waiting for admission, FIFO
        slot_req: Dict[int, tuple] = {}
        nxt = 0
        busy_s = 0.0
        conc = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        try:
            while len(results) < len(reqs):
                # arrivals -> host preparation
                while nxt < len(reqs) and reqs[nxt].arrival_s <= now():
                    r = reqs[nxt]
                    futures.append((r, ex.submit(Prepared, r.model_dir)))
                    nxt += 1
                # prepared (in arrival order) -> admission queue
                while futures and futures[0][1].done():
                    r, f = futures.pop(0)
                    ready.append((r, f.result()))
                # admit in FIFO order while slots and budget allow
                while ready:
                    r, prep = ready[0]
                    if prep.bytes > self.budget:
                        raise RuntimeError(f"request {r.rid} needs {prep.bytes} device bytes, above the budget")
                    k = self.pool.admit(prep, -1.0 if r.t_end is None else r.t_end)
                    if k < 0:
                        break
                    ready.pop(0)
                    slot_req[k] = (r, now())
                if slot_req:
                    tb = time.perf_counter()
                    running = self.pool.advance(self.chunk)
                    busy_s += time.perf_counter() - tb
                    conc.append(running)
                    for k in self.pool.finished():
                        r, ta = slot_req.pop(k)
                        s = self.pool.scalars(k)
                        fl = {name: self.pool.get(k, name) for name in fetch}
                        cells = self.pool.nps[k]
                        self.pool.release(k)
                        results.append(Result(r.rid, r.arrival_s, ta, now(), cells, int(s["nt"]), s["t"],
                                              int(s["error"]), fl))
                else:
                    # idle: wait for the next arrival or a preparation
                    time.sleep(0.002)
        finally:
            ex.shutdown(wait=True)
        makespan = max(r.done_s for r in results) - min(r.arrival_s for r in results)
        lat = np.array([r.latency_s for r in results])
        return {
            "results": sorted(results, key=lambda r: r.rid),
            "makespan_s": makespan,
            "scenarios_per_h": len(results) / makespan * 3600.0,
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_max_s": float(lat.max()),
            "device_busy_s": busy_s,
            "mean_running": float(np.mean(conc)) if conc else 0.0,
        }
