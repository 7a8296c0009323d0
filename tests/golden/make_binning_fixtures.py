"""Generate tests/golden/reference_binning.json: the trough example's receiver flux binning,
computed by the reference's own post-processing functions.

    SOLTRACE_REFERENCE=<reference checkout> python tests/golden/make_binning_fixtures.py

The example (app/deploy/api/examples/parabolic-trough-tracking-timeseries) bins absorbed
rays on the absorber tube by the nearest node of a polar mesh: convert_xy_polar_coords
(st_processing_functions.py:207-224) turns (x, z) into the arc position r atan2(x, z - f),
create_polar_mesh_cyl (174-204) lays nx x ny cell centres over the circumference and the
tube length, and compute_fluxmap (236-276) adds every ray to the node nearest in each
direction.  Its module imports plotting and solar-position packages at the top; they are
replaced by empty stand-ins (the binning uses numpy and pandas only).

Each case holds the tube radius r, the length l, nx, ny, element-local points (x, y, z) on
the tube (axis at z = r, so the example's focal height f is r and its z - f is exactly the
local z - r), and the count grid [ix][iy] that compute_fluxmap gives for them with a power
per ray of anode x 1000 (one unit of flux per ray).  The tests re-bin the points with the
oracle's kind-4 rule (tests/test_binning_kat.py).
"""
from __future__ import annotations

import io
import json
import math
import os
import sys
import types
from contextlib import redirect_stdout

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SOLTRACE_REFERENCE", "/root/reference")
EXAMPLE = os.path.join(REF, "app", "deploy", "api", "examples", "parabolic-trough-tracking-timeseries")


def _stub_modules():
    class _Any(types.ModuleType):
        def __getattr__(self, name):
            return _Any(name)

        def __call__(self, *a, **k):
            return _Any("call")

    for name in ["matplotlib", "matplotlib.pyplot", "pvlib", "pvlib.solarposition", "pvlib.tracking", "plotly",
                 "plotly.graph_objects", "plotly.io", "scipy", "scipy.interpolate"]:
        sys.modules[name] = _Any(name)


def _points(rng, r, l, n):
    th = rng.uniform(-math.pi, math.pi, n)
    y = rng.uniform(-0.6 * l, 0.6 * l, n)
    y[: min(8, n)] = [0.0, l / 2, -l / 2, 0.25 * l, -0.25 * l, 0.7 * l, -0.7 * l, 1e-12][: min(8, n)]
    pts = np.stack([r * np.sin(th), y, r + r * np.cos(th)], axis=1)
    pts[0] = [-r, 0.0, r]
    pts[1] = [0.0, 0.0, 0.0]
    pts[2] = [r, 0.0, r]
    return pts


def main():
    _stub_modules()
    sys.path.insert(0, EXAMPLE)
    import pandas as pd
    import st_processing_functions as spf

    rng = np.random.default_rng(20240611)
    cases = []
    r_kat = 1 / 28.5714
    for r, l, nx, ny, n in [(r_kat, 1.0, 5, 4, 3), (r_kat, 1.0, 5, 3, 3), (r_kat, 1.0, 5, 4, 400),
                            (0.035, 12.0, 72, 120, 1200), (0.035, 4.0, 1, 2, 50), (0.05, 2.0, 2, 1, 50),
                            (0.0125, 0.5, 17, 9, 300), (0.2, 7.0, 40, 40, 500)]:
        pts = _points(rng, r, l, n)
        d = r * 2.0
        Xc, Yc, xn, yn, dx, dy, psi = spf.create_polar_mesh_cyl(d, l, nx, ny)
        dfr = pd.DataFrame({"loc_x": pts[:, 0], "loc_y": pts[:, 1], "loc_z": pts[:, 2]})
        dfr["ypos"] = dfr.loc_y
        dfr["cpos"] = spf.convert_xy_polar_coords(d, dfr.loc_x, dfr.loc_z, r, gui_coords=True)
        with redirect_stdout(io.StringIO()):
            flux, _ = spf.compute_fluxmap(dx * dy * 1000.0, dfr, d, l, nx, ny)
        counts = np.rint(flux).astype(int)
        assert np.allclose(flux, counts, atol=1e-9) and counts.sum() == n
        cases.append({"r": r, "l": l, "nx": nx, "ny": ny, "points": pts.tolist(), "counts": counts.tolist(),
                      "x_nodes": [float(v) for v in xn], "y_nodes": [float(v) for v in yn]})
    with open(os.path.join(HERE, "reference_binning.json"), "w") as f:
        json.dump({"source": "st_processing_functions.py (trough example): create_polar_mesh_cyl, "
                             "convert_xy_polar_coords, compute_fluxmap", "cases": cases}, f)
    print(f"{len(cases)} cases")


if __name__ == "__main__":
    main()
