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
}

# Algorithmic bytes per cell-update of this layout (each element read or written
# once per kernel; stencil neighbours served from cache), wet faces in the table
# interpolation branch.  Derivation in DESIGN.md.
BYTES = {
    "subgrid": {"momentum": 125, "continuity": 67},
    "plain": {"momentum": 60, "continuity": 26},
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
    if kind == "subgrid":
        import torch

        dev = "cuda" if torch.cuda.is_available() else "cpu"
        m = synth.subgrid_regular(device=dev, **kw)
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


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
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
    # warm-up steps (untimed); graphs get instantiated here
    g.issue(max(args.warmup, 3))
    g.sync()
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
            traffic = json.load(open(tfile)).get("momentum_bytes_per_launch_scaled")
        except Exception:
            traffic = None
    s1 = g.scalars()
    # ---- full simulated run (12 h for the subgrid workload), device-resident
    full = None
    if args.full_run and rank == 0:
        g2 = Model(d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2.run(g2.scalars()["t1"], chunk=64)
        el = time.perf_counter() - t0
        sf = g2.scalars()
        full = {"simulated_s": sf["t"] - sf["t0"], "steps": int(sf["nt"]), "wall_s": el,
                "cell_updates_per_s": npc * sf["nt"] / el, "error_flag": int(sf["error"])}
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
        for _ in range(3):
            b.update()
        ksteps = max(10, min(args.steps, 100))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(ksteps):
            qext[:] = 0.0
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
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 time and volume)", "data": "synthetic",
        "config": {"workload": desc, "cells": npc, "global_cells": npc * world, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (device-resident state %.1f GB)" % (s0["device_bytes"] / 1e9),
                   "timed_from_t_s": s0["t"], "sim_time_after_timing_s": s1["t"]},
        "gpu_launches": lps * args.steps,
        "kernel_ms": {"step_bnd": ktimes[0], "momentum": ktimes[1], "sources": ktimes[2], "continuity": ktimes[3]},
        "roofline": {"bound": "hbm", "kernel": "k_momentum", "achieved": ach_mom, "peak": peak, "unit": "GB/s",
                     "frac": ach_mom / peak, "traffic": traffic, "peak_source": peak_src,
                     "bytes_per_cell": BYTES[wl], "step_achieved_gbs": step_bytes, "step_frac": step_bytes / peak},
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cb,
        "full_run": full,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="subgrid", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--full-run", type=int, default=1, help="also time the whole simulated period (rank 0)")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline work")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
