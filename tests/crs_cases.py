"""Cross-sections for the test models: a crs file (name line, "nrows ncols",
nrows lines of x y, as sfincs_crosssections.f90:8-127 reads it) added to a
model directory."""
import os

LINES = [("crs_east", [(6100.0, 500.0), (6100.0, 9000.0)]),            # crosses u faces
         ("'crs north'", [(2000.0, 4900.0), (10000.0, 4900.0)]),      # v faces; a quoted name
         ("diag", [(3000.0, 1000.0), (6000.0, 3000.0), (9000.0, 8000.0)])]


def add_crs(d, lines=LINES, scale=1.0):
    """The lines are laid out for a 12 km x 9.6 km grid; scale shrinks them."""
    with open(os.path.join(d, "sfincs.crs"), "w") as f:
        for name, pts in lines:
            f.write(f"{name}\n{len(pts)} 2\n")
            for x, y in pts:
                f.write(f"{x * scale:.1f} {y * scale:.1f}\n")
    with open(os.path.join(d, "sfincs.inp"), "a") as f:
        f.write(f"{'crsfile':<20} = sfincs.crs\n")


NAMES = ["crs_east", "crs north", "diag"]
