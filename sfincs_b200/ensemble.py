"""Uneven flood-scenario ensembles: member specifications and cached generation.

An ensemble member is a subgrid regular-grid model (the generator of
``synth.subgrid_regular``) with its own size, DEM seed, surge peak and rain
rate; a spec with ``kind="quadtree"`` is a quadtree mesh of
``qtsynth.quadtree_coastal`` instead.  The batched form advances all members with the same launches
(``bmi.Ensemble``); the plain form solves them one after another
(``bmi.Model``).
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import tempfile
import time
from typing import Dict, List

import numpy as np


def member_specs(n: int = 64, seed: int = 7, side_lo: int = 200, side_hi: int = 1500, dx: float = 100.0,
                 P: int = 10, tstop: float = 21600.0) -> List[Dict]:
    """n members with sides drawn log-uniformly from [side_lo, side_hi] cells,
    surge peaks U(1, 4) m and rain U(0, 80) mm/h (for the first half of the
    run), each simulating ``tstop`` seconds; seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        side = int(round(float(np.exp(rng.uniform(np.log(side_lo), np.log(side_hi))))))
        out.append(dict(nmax=side, mmax=side, dx=dx, P=P, seed=seed * 1000 + i, tstop=tstop,
                        surge_peak=float(rng.uniform(1.0, 4.0)), rain_mmh=float(rng.uniform(0.0, 80.0)),
                        rain_hours=tstop / 7200.0, coast_x=0.15 * side * dx, t_peak=tstop / 2, width_h=6.0))
    return out


def generate(specs: List[Dict], root: str = None, device: str = None, log=None) -> List[str]:
    """Write every member's model directory (cached under the temp dir by the
    hash of its spec) and return the directories."""
    from . import synth

    if device is None:
        try:
            import torch

            device = "cuda" if torch.cuda.is_available() else "cpu"
        except Exception:
            device = "cpu"
    root = root or tempfile.gettempdir()
    dirs = []
    t0 = time.time()
    for spec in specs:
        key = hashlib.sha1(json.dumps(spec, sort_keys=True).encode()).hexdigest()[:12]
        d = os.path.join(root, f"sfincs_b200_member_{key}")
        if not os.path.exists(os.path.join(d, "READY")):
            tmp = d + f".tmp{os.getpid()}"
            shutil.rmtree(tmp, ignore_errors=True)
            kw = dict(spec)
            if kw.pop("kind", "subgrid") == "quadtree":
                from . import qtsynth

                m = qtsynth.quadtree_coastal(device=device, **kw)
            else:
                m = synth.subgrid_regular(device=device, **kw)
            m.write(tmp)
            open(os.path.join(tmp, "READY"), "w").write("ok\n")
            shutil.rmtree(d, ignore_errors=True)
            os.replace(tmp, d)
        dirs.append(d)
    if device == "cuda":
        import torch

        torch.cuda.empty_cache()
    if log:
        log(f"ensemble of {len(dirs)} members ready in {time.time() - t0:.1f}s")
    return dirs
