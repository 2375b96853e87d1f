"""Gridded meteo inputs for the tests: seeded wind, pressure and rain series on
an equidistant grid around a model, written in the reference's ASCII format."""
import os

import numpy as np

from sfincs_b200 import synth


def add_meteo(d, x_ext, y_ext, seed=1, nt=7, dt_rec=900.0, wind=True, pres=True, rain=True, dtwnd=600.0,
              extra=None):
    """Write amu/amv/amp/ampr files covering [-1 km, x_ext + 1 km] x [-1 km,
    y_ext + 1 km] (a grid coarser than the model) and append their keys."""
    rng = np.random.default_rng(seed)
    nr, nc = 9, 11
    x_ll, y_ll = -1000.0, -1000.0
    dx = (x_ext + 2000.0) / (nc - 2)
    dy = (y_ext + 2000.0) / (nr - 2)
    t = np.arange(nt) * dt_rec
    keys = {"dtwnd": dtwnd}
    if wind:
        u = 12.0 + 6.0 * rng.standard_normal((nt, nr, nc))
        v = 4.0 * rng.standard_normal((nt, nr, nc))
        synth.write_meteo_grid(os.path.join(d, "sfincs.amu"), "x_wind", "m s-1", x_ll, y_ll, dx, dy, t, u)
        synth.write_meteo_grid(os.path.join(d, "sfincs.amv"), "y_wind", "m s-1", x_ll, y_ll, dx, dy, t, v)
        keys.update(amufile="sfincs.amu", amvfile="sfincs.amv")
    if pres:
        p = 101200.0 + 400.0 * rng.standard_normal((nt, nr, nc))
        synth.write_meteo_grid(os.path.join(d, "sfincs.amp"), "air_pressure", "Pa", x_ll, y_ll, dx, dy, t, p)
        keys.update(ampfile="sfincs.amp", pavbnd=101300.0)
    if rain:
        r = np.abs(30.0 * rng.standard_normal((nt, nr, nc)))
        synth.write_meteo_grid(os.path.join(d, "sfincs.ampr"), "precipitation", "mm/hr", x_ll, y_ll, dx, dy, t, r)
        keys.update(amprfile="sfincs.ampr")
    keys.update(extra or {})
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        for k, v in keys.items():
            f.write(f"{k:<20} = {v}\n")
    return dict(x_ll=x_ll, y_ll=y_ll, dx=dx, dy=dy, nr=nr, nc=nc, times=t,
                rain=r if rain else None)


def add_spiderweb(d, x_ext, y_ext, seed=2, nrows=12, ncols=18, t_first=600.0, dt_rec=900.0, nt=4, rain=25.0,
                  dtwnd=600.0, extra=None):
    """Write a seeded cyclone whose eye crosses the model from south-west to
    north-east (records from t_first, so the first window fades it in and the
    last fades it out) and append spwfile and its keys."""
    rng = np.random.default_rng(seed)
    radius = 1.2 * max(x_ext, y_ext)
    t = t_first + np.arange(nt) * dt_rec
    xe = np.linspace(0.1 * x_ext, 0.9 * x_ext, nt)
    ye = np.linspace(-0.2 * y_ext, 0.8 * y_ext, nt)
    c = synth.cyclone(rng, nt, nrows, ncols, rain=rain)
    synth.write_spiderweb(os.path.join(d, "sfincs.spw"), t, xe, ye, radius, c["vmag"], c["vdir"], c["pdrop"],
                          c.get("prcp"))
    keys = {"spwfile": "sfincs.spw", "dtwnd": dtwnd}
    keys.update(extra or {})
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        for k, v in keys.items():
            f.write(f"{k:<20} = {v}\n")
    return dict(times=t, xe=xe, ye=ye, radius=radius, nrows=nrows, ncols=ncols, **c)
