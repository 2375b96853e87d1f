"""Profiling driver: advance a synthetic workload by a few direct-launch steps.

Used as the target of ncu captures (ncu sees individual launches: one
k_step_bnd, one k_momentum, one k_continuity per step).  Example:

    python -m sfincs_b200.profile_run --workload subgrid --n 1000 --warmup 5 --steps 3
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="subgrid", choices=["subgrid", "plain", "quadtree"])
    ap.add_argument("--n", type=int, default=1000,
                    help="cells per side (subgrid), nmax (plain) or level-1 cells per side (quadtree)")
    ap.add_argument("--P", type=int, default=20, help="subgrid pixels per cell side")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--steps", type=int, default=3)
    args = ap.parse_args()
    import torch

    from sfincs_b200 import synth
    from sfincs_b200.bmi import Model

    d = os.path.join(tempfile.gettempdir(), f"sfincs_b200_prof_{args.workload}_{args.n}_{args.P}")
    if not os.path.exists(os.path.join(d, "sfincs.inp")):
        if args.workload == "subgrid":
            m = synth.subgrid_regular(nmax=args.n, mmax=args.n, dx=100.0, P=args.P, seed=2, tstop=43200.0,
                                      device="cuda")
        elif args.workload == "quadtree":
            from sfincs_b200 import qtsynth

            # the bench's quadtree workload scaled to n level-1 cells per side (800 in the bench)
            m = qtsynth.quadtree_coastal(nmax1=args.n, mmax1=args.n, dx1=400.0, nlev=4,
                                         bands=(6000.0, 4000.0, 2000.0), P=4, seed=3, tstop=21600.0, subgrid=True,
                                         walk_km=9000.0 * (args.n / 800.0) ** 2, device="cuda")
        else:
            m = synth.plain_regular(nmax=args.n, mmax=int(args.n * 1.25), dx=50.0)
        m.write(d)
        torch.cuda.empty_cache()
    g = Model(d)
    g.issue(args.warmup)
    g.sync()
    for _ in range(args.steps):
        g.issue(1)
    g.sync()
    s = g.scalars()
    print(f"np {int(s['np'])} nt {int(s['nt'])} t {s['t']:.2f} dt {s['dt']:.4f}")


if __name__ == "__main__":
    main()
