"""Runs the reference's pysoltrace front end, unmodified, in this process (used by
tests/test_pysoltrace.py, one fresh process per case).

    python tests/pysoltrace_driver.py <case> <work dir> <pysoltrace dir> <output .npz>

The work directory holds coretrace_api.so (pysoltrace loads it from the working directory,
pysoltrace.py:1518-1531).  pysoltrace imports matplotlib at the top (pysoltrace.py:5) and its
trace plot uses plotly; both are replaced by stand-ins, and the stand-in's contourf keeps the
array plot_flux draws: the flux map pysoltrace computes (pysoltrace.py:1916-1960).

Cases:
  dish   a parabolic dish and a flat receiver built through pysoltrace's objects, run with
         seed 123 in one thread; saves the ray table (PT.raydata), the sun statistics, the
         power per ray and plot_flux's 25 x 25 map, and writes the system with pysoltrace's
         own write_soltrace_input_file (dish.stinput) for the oracle to read back.
  tower  the reference's tower demo script (examples/tower-demo.py) as shipped: three
         heliostats and a flat receiver, 1e6 hits over 8 worker processes (seeds seed + i 123,
         ray numbers offset per worker, pysoltrace.py:1614-1662), then its input-file writer,
         trace plot and 50 x 50 flux map.
"""
import os
import runpy
import sys
import types

import numpy as np

CAPTURED = {}


class _Anything(types.ModuleType):
    """A module, class, function or value that accepts every use."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Anything(name)

    def __call__(self, *a, **k):
        return _Anything("result")

    def __iter__(self):
        return iter([_Anything("a"), _Anything("b")])


def _stub_plotting():
    plt = _Anything("matplotlib.pyplot")

    def contourf(*a, **k):
        CAPTURED["flux"] = np.array(a[2], dtype=np.float64)
        return _Anything("contour")

    plt.contourf = contourf
    mpl = _Anything("matplotlib")
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    for name in ("plotly", "plotly.graph_objects", "plotly.io", "plotly.express"):
        sys.modules[name] = _Anything(name)


def _dish(PySolTrace, Point):
    PT = PySolTrace()
    mirror = PT.add_optic("Mirror")
    mirror.front.reflectivity = 0.95
    mirror.front.slope_error = 2.0
    mirror.front.spec_error = 0.5
    absorber = PT.add_optic("Absorber")
    absorber.front.reflectivity = 0.0
    sun = PT.add_sun()
    sun.shape = "p"
    sun.sigma = 4.65
    sun.position = Point(0.0, 0.0, 100.0)
    st = PT.add_stage()
    dish = st.add_element()
    dish.optic = mirror
    dish.position = Point(0.0, 0.0, 0.0)
    dish.aim = Point(0.0, 0.0, 1.0)
    dish.surface_parabolic(5.0, 5.0)
    dish.aperture_circle(10.0)
    sr = PT.add_stage()
    rec = sr.add_element()
    rec.optic = absorber
    rec.position = Point(0.0, 0.0, 5.0)
    rec.aim = Point(0.0, 0.0, 0.0)
    rec.surface_flat()
    rec.aperture_rectangle(0.5, 0.5)
    PT.num_ray_hits = 20000
    PT.max_rays_traced = 2_000_000
    PT.is_sunshape = True
    PT.is_surface_errors = True
    res = PT.run(123, False, 1)
    PT.write_soltrace_input_file("dish.stinput")
    PT.plot_flux(rec, nx=25, ny=25, display=False)
    return PT, res


def main():
    case = sys.argv[1]
    work, pys_dir, out = (os.path.abspath(a) for a in sys.argv[2:5])
    os.chdir(work)
    _stub_plotting()
    sys.path.insert(0, pys_dir)
    if case == "dish":
        from pysoltrace import PySolTrace, Point
        PT, res = _dish(PySolTrace, Point)
    elif case == "tower":
        g = runpy.run_path(os.path.join(pys_dir, "examples", "tower-demo.py"), run_name="__main__")
        PT, res = g["PT"], 1
    else:
        raise SystemExit(f"unknown case {case}")
    df = PT.raydata
    np.savez(out, res=res, loc=df[["loc_x", "loc_y", "loc_z"]].to_numpy(),
             cos=df[["cos_x", "cos_y", "cos_z"]].to_numpy(), element=df["element"].to_numpy(),
             stage=df["stage"].to_numpy(), number=df["number"].to_numpy(), ppr=PT.powerperray,
             sun=np.array([PT.sunstats[k] for k in ("xmin", "xmax", "ymin", "ymax", "nsunrays")], dtype=np.float64),
             flux=CAPTURED.get("flux", np.zeros(0)))


if __name__ == "__main__":
    main()
