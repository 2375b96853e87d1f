"""Regenerates tests/golden/*.npz: small seeded cases and the FP64 oracle state
after a fixed number of steps.  The fixtures pin the oracle against regressions;
tests/golden/pyref.py (an independent pure-Python restatement) pins it against
the reference's formulas.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def cases():
    from sfincs_b200 import synth

    m = synth.plain_regular(nmax=6, mmax=8, dx=250.0, tstop=900.0, seed=11, nbumps=3)
    yield "plain_6x8", m, 40
    m = synth.subgrid_regular(nmax=8, mmax=10, dx=300.0, P=4, seed=12, tstop=1800.0, coast_x=900.0,
                              t_peak=900.0, width_h=0.3, surge_peak=1.0, rain_hours=0.2)
    yield "subgrid_8x10", m, 40


def main():
    from oracle.oracle import Oracle

    for name, m, nsteps in cases():
        d = tempfile.mkdtemp()
        m.write(d)
        o = Oracle(d, "fp64")
        o.update(-1000.0, nsteps)
        s = o.scalars()
        out = {"zs": o.get("zs"), "q": o.get("q"), "uv": o.get("uv"), "t": s["t"], "nt": s["nt"]}
        if s["subgrid"]:
            out["z_volume"] = o.get("z_volume")
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, int(s["nt"]), s["t"])


if __name__ == "__main__":
    main()
