"""Astronomic boundary cases: a .bca file (one [forcing] block per boundary
point, constituent name, amplitude in m, phase in degrees, in the layout of
the reference's reader, sfincs_boundaries.f90:289-450) added to a model
directory."""
import os


def write_bca(path, sets):
    """sets: per boundary point a list of (name, amplitude, phase)."""
    with open(path, "w") as f:
        for k, comps in enumerate(sets):
            f.write("[forcing]\n")
            f.write(f"Name                            = bnd_{k + 1:04d}\n")
            f.write("Function                        = astronomic\n")
            f.write("Quantity                        = astronomic component\n")
            f.write("Unit                            = -\n")
            f.write("Quantity                        = waterlevelbnd amplitude\n")
            f.write("Unit                            = m\n")
            f.write("Quantity                        = waterlevelbnd phase\n")
            f.write("Unit                            = deg\n")
            for name, a, p in comps:
                f.write(f"{name:<8s} {a:10.5f} {p:10.3f}\n")
            f.write("\n")


def add_bca(d, sets, extra=None):
    """Write sfincs.bca into model directory d and name it in sfincs.inp."""
    write_bca(os.path.join(d, "sfincs.bca"), sets)
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'bcafile':<20} = sfincs.bca\n")
        for k, v in (extra or {}).items():
            f.write(f"{k:<20} = {v}\n")


def set_tref(d, tref):
    """Replace tref, tstart and tstop in sfincs.inp, keeping the run length."""
    import datetime as dt

    p = os.path.join(d, "sfincs.inp")
    lines = open(p).read().splitlines()
    keys = {ln.split("=")[0].strip(): ln.split("=", 1)[1].strip() for ln in lines if "=" in ln}
    fmt = "%Y%m%d %H%M%S"
    t0 = dt.datetime.strptime(keys["tstart"], fmt)
    t1 = dt.datetime.strptime(keys["tstop"], fmt)
    new0 = dt.datetime.strptime(tref, fmt)
    repl = {"tref": tref, "tstart": tref, "tstop": (new0 + (t1 - t0)).strftime(fmt)}
    out = []
    for ln in lines:
        k = ln.split("=")[0].strip() if "=" in ln else None
        out.append(f"{k:<20} = {repl[k]}" if k in repl else ln)
    with open(p, "w") as f:
        f.write("\n".join(out) + "\n")


# Main constituents of global tide models (the set a typical bca carries).
MAIN = ["M2", "S2", "N2", "K2", "K1", "O1", "P1", "Q1", "MF", "MM", "M4", "MS4", "MN4"]
