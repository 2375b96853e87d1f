"""Benchmark of the B200 SFINCS time-stepping core.

Default workload (N=1): the subgrid regular grid of 2000 x 2000 computational
cells at 100 m (4M cells) with 10-level subgrid volume and uv tables built from
a seeded 5 m fractal DEM (Hurst 0.8, relief -15..+25 m, coastline at x=30 km),
a Gaussian surge hydrograph (3 m peak, 6 h FWHM) on the west boundary and
40 mm/h uniform rain for 3 h; 12 h simulated.  Inputs are synthetic (no public
benchmark data exists for this path); all state lives in HBM.

A "step" is one model time step of the whole grid (step control + boundary
forcing, momentum, continuity).  `value` is cell-updates/s with inputs resident
in HBM (CUDA events on the library's stream); `e2e` is the same metric through
the reference-facing BMI C-ABI (update() with a host qext array pushed and the
host zs array refreshed every step).

Multi-GPU (`--gpus N` under torchrun): replicas only -- every rank advances its
own copy of the workload; NCCL is used for the barrier and the max-over-ranks
time, never on the data path.

`--impl reference` times the reference-semantics CPU restatement (the oracle in
the reference's mixed precision, OpenMP over all host cores): the Fortran
reference itself cannot be compiled in this image.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (builder kwargs, description)
    "subgrid": (dict(kind="subgrid", nmax=2000, mmax=2000, dx=100.0, P=20, seed=2, tstop=43200.0),
                "subgrid regular grid 2000x2000 @100 m (4M cells), 10-level tables from a 5 m fractal DEM, "
                "3 m surge + 40 mm/h rain 3 h, 12 h simulated"),
    "plain": (dict(kind="plain", nmax=400, mmax=500, dx=50.0, seed=1, tstop=3600.0),
              "plain regular grid 500x400 @50 m (200k cells), 1:100 beach + 20 bumps, 1 m tide, 1 h simulated"),
    "quadtree": (dict(kind="quadtree", nmax1=800, mmax1=800, dx1=400.0, nlev=4, bands=(6000.0, 4000.0, 2000.0), P=4,
                      seed=3, tstop=21600.0, subgrid=True, walk_km=9000.0, tide_amp=1.5, tide_period=44712.0,
                      wind_speed=30.0, advection=1, viscosity=1),
                 "quadtree 4 levels 400 m -> 50 m (~8.1M cells) refined within 2/4/6 km of a seeded 9000 km "
                 "random-walk polyline in a 320 km box, 10-level subgrid tables (12.5 m DEM), advection + viscosity, "
                 "30 m/s onshore wind, 1.5 m 12.42 h tide, 6 h simulated"),
}

# Algorithmic bytes per cell-update of this layout (each element read or written
# once per kernel; stencil neighbours served from cache), every face wet: the
# subgrid table values reach a face through its 24-byte record-cache entry, so
# a level change adds one table record read and one entry write.
BYTES = {
    "subgrid": {"momentum": 111, "continuity": 76},
    "plain": {"momentum": 60, "continuity": 26},
    "quadtree": {"momentum": 219, "continuity": 83},
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_dir(name: str, rank: int) -> str:
    """Generate (or reuse from /tmp) the model directory of a named workload."""
    kw, _ = WORKLOADS[name]
    key = hashlib.sha1(json.dumps(kw, sort_keys=True).encode()).hexdigest()[:12]
    d = os.path.join(tempfile.gettempdir(), f"sfincs_b200_bench_{name}_{key}")
    if os.path.exists(os.path.join(d, "READY")):
        return d
    lock = d + ".lock"
    if rank != 0:  # rank 0 generates, the others wait for it (same box)
        t0 = time.time()
        while not os.path.exists(os.path.join(d, "READY")):
            if time.time() - t0 > 1800:
                raise RuntimeError("timed out waiting for the workload to be generated")
            time.sleep(1.0)
        return d
    from sfincs_b200 import synth

    t0 = time.time()
    tmp = d + f".tmp{os.getpid()}"
    shutil.rmtree(tmp, ignore_errors=True)
    kw = dict(kw)
    kind = kw.pop("kind")
    if kind in ("subgrid", "quadtree"):
        import torch

        dev = "cuda" if torch.cuda.is_available() else "cpu"
        if kind == "subgrid":
            m = synth.subgrid_regular(device=dev, **kw)
        else:
            from sfincs_b200 import qtsynth

            m = qtsynth.quadtree_coastal(device=dev, **kw)
        if dev == "cuda":
            torch.cuda.empty_cache()
    else:
        m = synth.plain_regular(**kw)
    m.write(tmp)
    open(os.path.join(tmp, "READY"), "w").write("ok\n")
    shutil.rmtree(d, ignore_errors=True)
    os.replace(tmp, d)
    log(f"generated workload {name} in {time.time() - t0:.1f}s -> {d}")
    return d


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=self.f, stderr=subprocess.DEVNULL)
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    from sfincs_b200 import replicas

    return replicas.allreduce_max(x) if world > 1 else x


def barrier(world: int):
    if world > 1:
        from sfincs_b200 import replicas

        replicas.barrier()


def cpu_reference(d: str, steps: int, warmup: int, budget_s: float = 20.0):
    """Time the reference-semantics CPU restatement (oracle, 'ref' precision) on d."""
    from oracle.oracle import Oracle

    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    t0 = time.time()
    o = Oracle(d, "ref")
    t_init = time.time() - t0
    npc = o.scalars()["np"]
    o.update(-1000.0, max(1, warmup))
    t0 = time.perf_counter()
    o.update(-1000.0, 2)
    per = (time.perf_counter() - t0) / 2
    n = int(max(2, min(steps, budget_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    done = o.update(-1000.0, n)
    el = time.perf_counter() - t0
    o.close()
    return {"value": npc * done / el, "unit": "cell-updates/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port",
            "sample": f"{done} steps of the full {int(npc)}-cell workload after {max(1, warmup) + 2} warm-up steps "
                      f"(init {t_init:.1f}s excluded); OpenMP reference-precision restatement of the Fortran loops",
            "seconds": el}


def reference_scenarios(args):
    """Reference arm for the ensemble workload: the oracle (reference
    precision, all host cores) timed on a bounded sample of one mid-size
    member, extrapolated to every member's cell count and step count."""
    from oracle.oracle import Oracle
    from sfincs_b200 import ensemble

    specs = ensemble.member_specs(n=args.members)
    cells = np.array([s["nmax"] * s["mmax"] for s in specs], dtype=np.float64)
    mid = int(np.argsort(cells)[len(specs) // 2])
    d = ensemble.generate([specs[mid]], log=log)[0]
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    o = Oracle(d, "ref")
    npc = o.scalars()["np"]
    o.update(-1000.0, 5)
    t0 = time.perf_counter()
    done = 0
    while time.perf_counter() - t0 < args.cpu_budget:
        done += o.update(-1000.0, 5)
    el = time.perf_counter() - t0
    dt = o.scalars()["dt"]
    o.close()
    rate = npc * done / el
    tsim = specs[mid]["tstop"]
    total_s = float(np.sum(cells * (tsim / dt))) / rate
    value = len(specs) / total_s * 3600.0
    return {"impl": "reference", "metric": "scenarios/h", "value": value, "unit": "scenarios/h",
            "n_gpus": args.gpus, "steps": done, "warmup": 5, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 (reference precision)", "data": "synthetic",
            "config": {"workload": f"uneven ensemble of {len(specs)} members (as --workload ensemble)",
                       "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": value, "unit": "scenarios/h", "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": "port",
                             "sample": f"{done} steps of a {int(npc)}-cell member in {el:.1f}s "
                                       f"({rate:.3e} cell-updates/s), extrapolated to all members at dt={dt:.3f}s"},
            "e2e": {"value": value, "unit": "scenarios/h", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    if args.workload in ("ensemble", "serve"):
        print(json.dumps(reference_scenarios(args)), flush=True)
        return
    d = workload_dir(args.workload, rank)
    cb = cpu_reference(d, args.steps, args.warmup, budget_s=args.cpu_budget)
    _, desc = WORKLOADS[args.workload]
    line = {"impl": "reference", "metric": "cell-updates/s", "value": cb["value"], "unit": "cell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (reference precision)", "data": "synthetic",
            "config": {"workload": desc, "parallelism": "host OpenMP"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local: int):
    import torch

    from sfincs_b200.bmi import BMI, Model

    torch.cuda.set_device(local)
    d = workload_dir(args.workload, rank)
    barrier(world)
    g = Model(d)
    s0 = g.scalars()
    npc = int(s0["np"])
    stream = torch.cuda.ExternalStream(g.stream)
    # warm-up steps (untimed): W direct steps, then one 32-step CUDA-graph chunk so
    # that the graph is captured and instantiated before the timed region
    warm = max(args.warmup, 3) + 32
    g.issue(max(args.warmup, 3))
    g.issue(32)
    g.sync()
    s_timed = g.scalars()  # state at the start of the timed region
    # ---- timed region: K steps, inputs resident in HBM (> L2: 3+ GB resident state)
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.issue(args.steps)
    e1.record(stream)
    g.sync()
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, world)
    ms_step = ms / args.steps
    value = world * npc * args.steps / (ms / 1e3)
    # ---- per-kernel durations (events between launches, same stream)
    ktimes, lps = g.kernel_times(max(20, min(args.steps, 100)))
    wl = args.workload
    bmom = BYTES[wl]["momentum"] * npc
    bcont = BYTES[wl]["continuity"] * npc
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    ach_mom = bmom / (ktimes[1] * 1e-3) / 1e9
    step_bytes = (bmom + bcont) / (ms_step * 1e-3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"traffic_{wl}.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get("momentum_bytes_per_launch")
        except Exception:
            traffic = None
    s1 = g.scalars()
    mom_kernel = "k_momentum" if os.environ.get("SFG_MOMENTUM_VARIANT", "5") in ("2", "3") else "k_momentum_tma"
    if wl == "quadtree":
        mom_kernel = "k_qt_momentum"
    # ---- full simulated run (12 h for the subgrid workload), device-resident
    full = None
    if args.full_run and rank == 0:
        g2 = Model(d)
        v0 = g2.volume()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2.run(g2.scalars()["t1"], chunk=64)
        el = time.perf_counter() - t0
        sf = g2.scalars()
        v1 = g2.volume()
        acc = sf["bflux_vol"] + sf["rain_vol"] + sf["src_vol"]
        full = {"simulated_s": sf["t"] - sf["t0"], "steps": int(sf["nt"]), "wall_s": el,
                "cell_updates_per_s": npc * sf["nt"] / el, "error_flag": int(sf["error"]),
                "volume_start_m3": v0, "volume_end_m3": v1, "volume_accounted_m3": acc,
                "volume_balance_rel": abs((v1 - v0) - acc) / max(abs(v1), 1.0)}
        del g2
    del g
    torch.cuda.empty_cache()
    # ---- end to end through the BMI C-ABI with host buffers
    e2e = None
    if rank == 0 or world > 1:
        b = BMI()
        b.initialize(d)
        qext = b.get_value_ptr("qext")  # host float[np], pushed to the device before every update
        zs = b.get_value_ptr("zs")      # host double[np], refreshed after every update
        qext[:] = 0.0  # the step's external source term, pushed to the device by every update()
        for _ in range(3):
            b.update()
        ksteps = max(10, min(args.steps, 100))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(ksteps):
            b.update()
            _ = float(zs[npc // 2])
        el = time.perf_counter() - t0
        el = max_over_ranks(el, world)
        b.finalize()
        e2e = {"value": world * npc * ksteps / el, "unit": "cell-updates/s", "h2d_bytes_per_step": npc * 4,
               "d2h_bytes_per_step": npc * 8, "steps": ksteps,
               "path": "BMI update() per step; host qext pushed (H2D) and host zs refreshed (D2H) every step"}
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cb = cpu_reference(d, args.steps, args.warmup, budget_s=args.cpu_budget)
        except Exception as ex:  # report, never fall back
            cb = {"value": None, "error": str(ex)}
    _, desc = WORKLOADS[wl]
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "graph_warmup_steps": warm - args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 time and volume)", "data": "synthetic",
        "config": {"workload": desc, "cells": npc, "global_cells": npc * world, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (device-resident state %.1f GB)" % (s0["device_bytes"] / 1e9),
                   "timed_from_t_s": s_timed["t"], "timed_from_step": int(s_timed["nt"]),
                   "sim_time_after_timing_s": s1["t"]},
        "gpu_launches": lps * args.steps,
        "kernel_ms": {"step_bnd": ktimes[0], "momentum": ktimes[1], "sources": ktimes[2], "continuity": ktimes[3],
                      "note": "each kernel timed alone with events around its own launches; in the graph the "
                              "launches overlap (programmatic dependent launch), so the sum exceeds ms_per_step"},
        "roofline": {"bound": "hbm", "kernel": mom_kernel, "achieved": ach_mom, "peak": peak, "unit": "GB/s",
                     "frac": ach_mom / peak, "traffic": traffic, "peak_source": peak_src,
                     "bytes_per_cell": BYTES[wl], "step_achieved_gbs": step_bytes, "step_frac": step_bytes / peak},
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cb,
        "full_run": full,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_ensemble(args, rank: int, world: int, local: int):
    """Uneven ensemble: 64 subgrid members (sides log-uniform 200..1500 cells),
    each simulating 6 h.  Batched (one launch sequence advances every member,
    per-member dt, CUDA graphs, autotuned kernel variant) against the plain
    path (the same members solved one after another, each with its own model).
    Members are split across ranks (replicas)."""
    import torch

    from sfincs_b200 import ensemble
    from sfincs_b200.bmi import Ensemble, Model

    torch.cuda.set_device(local)
    specs = ensemble.member_specs(n=args.members)
    mine = specs[rank::world]
    dirs = ensemble.generate(mine, log=log)
    barrier(world)
    ncell = [s["nmax"] * s["mmax"] for s in mine]
    # ---- batched
    E = Ensemble(dirs)
    E.set_autotune(True)
    t1 = [E.scalars(i)["t1"] for i in range(len(dirs))]
    st = torch.cuda.ExternalStream(E.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(world)
    e0.record(st)
    E.run(t1)
    e1.record(st)
    e1.synchronize()
    ms_b = max_over_ranks(e0.elapsed_time(e1), world)
    steps_b = [int(E.scalars(i)["nt"]) for i in range(len(dirs))]
    variant = E.variant
    zs_b = [E.get(i, "zs") for i in range(len(dirs))]
    E.close()
    torch.cuda.empty_cache()
    # ---- plain: one model at a time
    ms_p = 0.0
    ms_each = []
    same = True
    for i, d in enumerate(dirs):
        g = Model(d)
        sp = torch.cuda.ExternalStream(g.stream)
        torch.cuda.synchronize()
        e0.record(sp)
        g.run(g.scalars()["t1"])
        e1.record(sp)
        e1.synchronize()
        ms_each.append(e0.elapsed_time(e1))
        ms_p += ms_each[-1]
        same = same and np.array_equal(g.get("zs"), zs_b[i])
        g.close()
    ms_p = max_over_ranks(ms_p, world)
    # Where batching stands: the members' step counts differ (per-member dt);
    # a batched run cannot finish before its longest member alone, so
    # plain_sum / longest_alone bounds batched_over_plain for any batching.
    longest = int(np.argmax(ms_each))
    bound = ms_p / ms_each[longest]
    n_all = len(specs)
    value = n_all / (ms_b / 1e3) * 3600.0
    plain = n_all / (ms_p / 1e3) * 3600.0
    cell_updates = sum(c * s for c, s in zip(ncell, steps_b))
    line = {
        "metric": "scenarios/h", "value": value, "unit": "scenarios/h", "n_gpus": world, "steps": max(steps_b),
        "warmup": 0, "ms_per_step": ms_b / max(steps_b), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (f64 time and volume)", "data": "synthetic",
        "config": {"workload": f"uneven ensemble: {n_all} subgrid members, sides log-uniform 200..1500 cells at "
                               "100 m (P=10 subgrid pixels), surge U(1,4) m, rain U(0,80) mm/h, 6 h simulated each",
                   "members": n_all, "members_per_rank": len(dirs), "cells_total_rank0": int(sum(ncell)),
                   "parallelism": f"replicas x{world} (members split across ranks)",
                   "l2": "device-resident state far larger than L2"},
        "gpu_launches": None,
        "batched": {"seconds": ms_b / 1e3, "scenarios_per_h": value, "autotuned_variant": variant,
                    "cell_updates_per_s": cell_updates / (ms_b / 1e3)},
        "plain": {"seconds": ms_p / 1e3, "scenarios_per_h": plain},
        "batched_over_plain": value / plain,
        "alone_equals_mix_bitwise": bool(same),
        "members": {"cells": [int(c) for c in ncell], "steps": steps_b, "plain_ms": [round(x, 3) for x in ms_each]},
        "longest_member": {"cells": int(ncell[longest]), "steps": int(steps_b[longest]),
                           "alone_s": ms_each[longest] / 1e3,
                           "share_of_batched_time": ms_each[longest] / ms_b},
        "batched_over_plain_bound": bound,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_serve(args, rank: int, world: int, local: int):
    """Served forecast stream: requests (subgrid regular grids, lognormal sizes
    clipped to 0.1M..10M cells, seeded fractal DEMs, random surge and rain,
    24 h simulated each) arrive as a Poisson process whose rate loads the GPU
    to about 80 %; the continuous-batching server admits them by HBM budget
    and reports scenarios/h with p50/p99 latency.  Each rank serves its own
    stream (replicas)."""
    import torch

    from sfincs_b200 import ensemble
    from sfincs_b200.bmi import Model
    from sfincs_b200.serve import Request, Server

    torch.cuda.set_device(local)
    rng = np.random.default_rng(11 + rank)
    specs = []
    for i in range(args.requests):
        cells = float(np.clip(rng.lognormal(np.log(0.5e6), 1.0), 0.1e6, 10e6))
        seed = 5000 + 100 * rank + i
        if i % 3 == 2:  # every third request a 3-level quadtree mesh (about 4.7 cells per level-1 cell)
            n1 = max(40, int(round(np.sqrt(cells / 4.7))))
            specs.append(dict(kind="quadtree", nmax1=n1, mmax1=n1, dx1=400.0, nlev=3, bands=(4000.0, 2000.0), P=4,
                              seed=seed, tstop=86400.0, subgrid=True, walk_km=9000.0 * (n1 / 800.0) ** 2,
                              tide_amp=float(rng.uniform(0.5, 2.0)), wind_speed=float(rng.uniform(0.0, 30.0))))
        else:
            side = int(round(np.sqrt(cells)))
            specs.append(dict(nmax=side, mmax=side, dx=100.0, P=8, seed=seed, tstop=86400.0,
                              surge_peak=float(rng.uniform(1.0, 4.0)), rain_mmh=float(rng.uniform(0.0, 80.0)),
                              rain_hours=3.0, coast_x=0.15 * side * 100.0, t_peak=43200.0, width_h=6.0))
    dirs = ensemble.generate(specs, log=log)
    # calibration: device throughput and dt of a mid-size request of each kind -> service-time estimates
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kinds = [s.get("kind", "subgrid") for s in specs]
    cal = {}
    for kind in sorted(set(kinds)):
        idx = [i for i, k in enumerate(kinds) if k == kind]
        sizes = [specs[i]["nmax"] * specs[i]["mmax"] if kind != "quadtree" else specs[i]["nmax1"] ** 2 for i in idx]
        mid = idx[int(np.argsort(sizes)[len(idx) // 2])]
        g = Model(dirs[mid])
        g.step(64)
        st = torch.cuda.ExternalStream(g.stream)
        e0.record(st)
        g.issue(128)
        e1.record(st)
        e1.synchronize()
        cal[kind] = (g.scalars()["np"] * 128 / (e0.elapsed_time(e1) / 1e3), g.scalars()["dt"])
        g.close()
    cells_of = {}
    for i, d in enumerate(dirs):
        from sfincs_b200.serve import Prepared

        pr = Prepared(d)
        cells_of[i] = pr.cells
        pr.release()
    service = np.array([cells_of[i] * (86400.0 / cal[kinds[i]][1]) / cal[kinds[i]][0] for i in range(len(specs))])
    lam = 0.8 / service.mean()
    arrivals = np.cumsum(rng.exponential(1.0 / lam, size=len(specs)))
    arrivals -= arrivals[0]
    reqs = [Request(arrival_s=float(a), model_dir=d, rid=i) for i, (a, d) in enumerate(zip(arrivals, dirs))]
    torch.cuda.empty_cache()
    srv = Server(max_slots=32, chunk=32, prep_threads=4)
    barrier(world)
    out = srv.serve(reqs, fetch=("zsmax",))
    srv.close()
    torch.cuda.empty_cache()
    # each request alone on the idle device, for the cost of sharing it
    alone = {}
    for r in reqs:
        g = Model(r.model_dir)
        st = torch.cuda.ExternalStream(g.stream)
        e0.record(st)
        g.run(g.scalars()["t1"])
        e1.record(st)
        e1.synchronize()
        alone[r.rid] = e0.elapsed_time(e1) / 1e3
        g.close()
    served = {x.rid: x.latency_s for x in out["results"]}
    slow = np.array([served[k] / alone[k] for k in alone])
    makespan = max_over_ranks(out["makespan_s"], world)
    value = world * len(reqs) / makespan * 3600.0
    cells = [r.cells for r in out["results"]]
    cu = sum(r.cells * r.steps for r in out["results"])
    line = {
        "metric": "scenarios/h", "value": value, "unit": "scenarios/h", "n_gpus": world,
        "steps": int(sum(r.steps for r in out["results"])), "warmup": 0, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 time and volume)",
        "data": "synthetic",
        "config": {"workload": "served forecast stream: lognormal sizes (median 0.5M, clipped 0.1M..10M cells); "
                               "two of three requests subgrid regular grids at 100 m (P=8, surge U(1,4) m, rain "
                               "U(0,80) mm/h 3 h), one of three 3-level quadtree meshes (400 m -> 100 m, 10-level "
                               "subgrid tables, tide U(0.5,2) m, onshore wind U(0,30) m/s); 24 h simulated each; "
                               "Poisson arrivals at ~80 % estimated load",
                   "requests_per_rank": len(reqs), "quadtree_requests": int(sum(k == "quadtree" for k in kinds)),
                   "cells_min": int(min(cells)), "cells_max": int(max(cells)),
                   "arrival_rate_per_s": lam, "service_estimate_s": float(service.mean()),
                   "parallelism": f"replicas x{world} (one request stream per rank)"},
        "gpu_launches": None,
        "latency_p50_s": out["latency_p50_s"], "latency_p99_s": out["latency_p99_s"],
        "latency_max_s": out["latency_max_s"], "makespan_s": makespan, "mean_running": out["mean_running"],
        "alone_p50_s": float(np.percentile(list(alone.values()), 50)),
        "alone_p99_s": float(np.percentile(list(alone.values()), 99)),
        "served_over_alone_mean": float(slow.mean()), "served_over_alone_p99": float(np.percentile(slow, 99)),
        "alone_sum_s": float(sum(alone.values())),
        "cell_updates_per_s": cu / out["makespan_s"],
        "errors": int(sum(1 for r in out["results"] if r.error)),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="subgrid", choices=sorted(WORKLOADS) + ["ensemble", "serve"])
    ap.add_argument("--requests", type=int, default=30, help="requests per rank (--workload serve)")
    ap.add_argument("--members", type=int, default=64, help="ensemble members (--workload ensemble)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--full-run", type=int, default=1, help="also time the whole simulated period (rank 0)")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline work")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world)
        elif args.workload == "ensemble":
            run_ensemble(args, rank, world, local)
        elif args.workload == "serve":
            run_serve(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
