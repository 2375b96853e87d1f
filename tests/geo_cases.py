"""Geographic (crsgeo = 1) versions of the synthetic test models: the grid
spacing in degrees, chosen so that a cell at the model's reference latitude
has the projected model's size in metres."""
import math

import numpy as np

R = 111111.1  # metres per degree (sfincs_domain.f90:1416)


def geographic(m, lon0=4.0, lat0=40.0):
    """Turn a projected RegularModel into the same grid on longitude /
    latitude (boundary points converted too); returns the model."""
    c = math.cos(math.radians(lat0))
    dx_m, dy_m = m.dx, m.dy
    m.dx = dx_m / (R * c)
    m.dy = dy_m / R
    m.x0, m.y0 = lon0, lat0
    if m.bnd is not None:
        b = np.asarray(m.bnd, np.float64).copy()
        b[:, 0] = lon0 + b[:, 0] / (R * c)
        b[:, 1] = lat0 + b[:, 1] / R
        m.bnd = b
    m.params["crsgeo"] = 1
    return m
