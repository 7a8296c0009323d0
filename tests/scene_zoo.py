"""Small scenes that between them exercise every surface type, aperture shape,
sunshape, optical distribution, property table and stage flag of the trace.

Each scene is a few elements lit by a sun along -z; they are parity cases,
sized so that the CPU oracle and the reference finish in well under a second.
Surface-file scenes write synthetic .mon/.ply/.csi/.sht files into `tmpdir`.
"""
from __future__ import annotations

import math
import os

import numpy as np

from soltrace_b200.scenes import Element, OpticFace, OpticSet, Scene, Stage, Sun

MIRROR = OpticSet("mirror", OpticFace("g", refl=0.93, slope=1.5, spec=0.4), OpticFace("g", refl=0.93, slope=1.5, spec=0.4))
PERFECT = OpticSet("perfect", OpticFace("g", refl=1.0), OpticFace("g", refl=1.0))
TARGET = OpticSet("target", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0))


def _target(z=6.0, size=30.0):
    return Element(origin=(0, 0, z), aim=(0, 0, 0), aperture="r", aperture_params=(size, size), surface="f",
                   interaction=2, optic="target")


def _two_stage(elements, sun=None, optics=None, n=3000, target_z=6.0, **kw) -> Scene:
    optics = optics or [MIRROR, TARGET]
    sun = sun or Sun("p", 4.65, (0.0, 0.0, 100.0))
    return Scene(sun, optics, [Stage(elements, **kw), Stage([_target(target_z)])], raycount=n, raymax=200 * n + 10000)


def write_mon(path, focal=2.0):
    # z = x^2/(4f) + y^2/(4f): B(2,0) and B(2,2) (order 2, rows k=0..2, m=0..k)
    c = 1.0 / (4.0 * focal)
    vals = [2, 0.0, 0.0, 0.0, c, 0.0, c]
    with open(path, "w") as f:
        f.write("\n".join(str(v) for v in vals) + "\n")


def write_ply(path, focal=2.0):
    with open(path, "w") as f:
        f.write("3\n0\n0\n%r\n0.001\n" % (1.0 / (4.0 * focal)))


def write_csi(path, focal=2.0, r_in=0.2, r_out=2.2, n=15):
    r = np.linspace(r_in, r_out, n)
    z = r * r / (4.0 * focal)
    with open(path, "w") as f:
        f.write(f"{n}\n")
        for a, b in zip(r, z):
            f.write(f"{a:.6f}\t{b:.6f}\n")
        f.write(f"{r_in / (2 * focal):.6f}\t{r_out / (2 * focal):.6f}\n")


def write_sht(path, focal=2.0, n=400, seed=5):
    rng = np.random.default_rng(seed)
    c = 1.0 / (4.0 * focal)
    rad = 2.0
    pts = []
    while len(pts) < n:
        x, y = rng.uniform(-rad, rad, 2)
        if x * x + y * y <= rad * rad:
            pts.append((x, y))
    with open(path, "w") as f:
        f.write("Title line\n")
        f.write(f"{rad} {focal} 0\n")
        f.write(f"0 2 {n}\n")
        f.write("0 0\n")
        for v in [0.0, 0.0, 0.0, c, 0.0, c]:
            f.write(f"{v!r}\n")
        for x, y in pts:
            sx = math.atan(2 * c * x) + 0.0005 * rng.normal()
            sy = math.atan(2 * c * y) + 0.0005 * rng.normal()
            f.write(f"{x:.6f} {y:.6f} {sx:.8f} {sy:.8f} 0\n")


def write_fed(path, focal=2.0, half=3.5, side=30, seed=7):
    # finite-element nodes of a paraboloid z = r^2/(4f) on a jittered square grid reaching well
    # past the aperture, so that every zone of the nodes' bounding box has nodes around it
    # (a query in a zone with fewer than 3 nodes nearby makes the reference throw)
    rng = np.random.default_rng(seed)
    c = 1.0 / (4.0 * focal)
    g = np.linspace(-half, half, side)
    pts = []
    for x in g:
        for y in g:
            x1, y1 = x + rng.uniform(-0.2, 0.2) * (g[1] - g[0]), y + rng.uniform(-0.2, 0.2) * (g[1] - g[0])
            pts.append((x1, y1, c * (x1 * x1 + y1 * y1)))
    with open(path, "w") as f:
        f.write("fe surface\n")
        f.write(f"{len(pts)}\n")
        for x, y, z in pts:
            f.write(f"{float(x)!r} {float(y)!r} {float(z)!r}\n")


def zoo(tmpdir: str) -> dict:
    """name -> Scene"""
    os.makedirs(tmpdir, exist_ok=True)
    mon, ply, csi, sht = (os.path.join(tmpdir, n) for n in ("z.mon", "p.ply", "s.csi", "v.sht"))
    write_mon(mon)
    write_ply(ply)
    write_csi(csi)
    write_sht(sht)
    P = dict(origin=(0, 0, 0), aim=(0, 0, 1), interaction=2, optic="mirror")
    S = {}
    S["sphere_circle"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="s", surface_params=(0.1,), **P)])
    S["sphere_line"] = _two_stage([Element(aperture="l", aperture_params=(-1.5, 1.5, 3.0), surface="s",
                                           surface_params=(0.1,), **P)])
    S["hyperboloid"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="o",
                                           surface_params=(0.12, -0.69), **P)])
    S["ellipsoid"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="o",
                                         surface_params=(0.12, 0.5), **P)])
    S["parabola_hex"] = _two_stage([Element(aperture="h", aperture_params=(4.0,), surface="p",
                                            surface_params=(0.125, 0.125), **P)])
    S["parabola_tri"] = _two_stage([Element(aperture="t", aperture_params=(4.0,), surface="p",
                                            surface_params=(0.125, 0.125), **P)])
    S["parabola_rect"] = _two_stage([Element(aperture="r", aperture_params=(4.0, 3.0), surface="p",
                                             surface_params=(0.125, 0.1), **P)])
    S["parabola_annulus"] = _two_stage([Element(aperture="a", aperture_params=(0.5, 2.0, 270.0), surface="p",
                                                surface_params=(0.125, 0.125), **P)])
    S["parabola_irrtri"] = _two_stage([Element(aperture="i", aperture_params=(-2, -1.5, 2, -1, 0.3, 2), surface="p",
                                               surface_params=(0.125, 0.125), **P)])
    S["parabola_quad"] = _two_stage([Element(aperture="q", aperture_params=(-2, -2, 2, -1.5, 1.5, 2, -1.8, 1.6),
                                             surface="p", surface_params=(0.125, 0.125), **P)])
    S["trough_line"] = _two_stage([Element(aperture="l", aperture_params=(-2, 2, 3), surface="p",
                                           surface_params=(0.2, 0.0), **P)])
    S["cone"] = _two_stage([Element(aperture="c", aperture_params=(3.0,), surface="c", surface_params=(60.0,), **P)])
    S["general"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="g",
                                       surface_params=(0.12, 0.12, -0.3), **P)])
    S["flat_circle"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="f", **P)])
    # A torus lit straight from the sun box (rays start 10 km away) loses every root
    # to cancellation in the quartic, in the reference as well; feed it from a
    # virtual plane 3 m above instead.
    def torus_scene(angle):
        plane = Element(origin=(0, 0, 3.0), aim=(0, 0, 4.0), aperture="r", aperture_params=(5, 5), surface="f",
                        interaction=2, optic="mirror")
        tor = Element(aperture="a", aperture_params=(0.0, 0.0, angle), surface="d", surface_params=(1.5, 0.4), **P)
        return Scene(Sun("p", 4.65, (0.0, 0.0, 100.0)), [MIRROR, TARGET],
                     [Stage([plane], virtual=True), Stage([tor]), Stage([_target()])], raycount=3000,
                     raymax=1_000_000)
    S["torus"] = torus_scene(360.0)
    S["torus_sector"] = torus_scene(200.0)
    S["cylinder"] = _two_stage([Element(origin=(0, 0, -0.5), aim=(0, 0, 1), aperture="l", aperture_params=(0, 0, 4),
                                        surface="t", surface_params=(2.0,), interaction=2, optic="mirror")])
    S["zernike"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="m", surface_file=mon, **P)])
    S["poly"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="r", surface_file=ply, **P)])
    S["spline"] = _two_stage([Element(aperture="a", aperture_params=(0.3, 2.1, 360.0), surface="i", surface_file=csi,
                                      **P)])
    S["vshot"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="v", surface_file=sht, **P)],
                            n=1500)
    # sunshapes and optical distributions
    t = np.linspace(0, 20, 30)
    inten = np.where(t < 4.65, 1.0, 0.05 * np.exp(-(t - 4.65) / 4.0))
    dish = Element(aperture="c", aperture_params=(4.0,), surface="p", surface_params=(0.125, 0.125), **P)
    fed = os.path.join(tmpdir, "dish.fed")
    write_fed(fed)
    S["fe_surface"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="e", surface_file=fed, **P)])
    S["sun_gauss"] = _two_stage([dish], sun=Sun("g", 2.5, (0.0, 0.0, 100.0)))
    S["sun_table"] = _two_stage([dish], sun=Sun("d", 0.0, (0.0, 0.0, 100.0), table=(t, inten)))
    S["sun_point"] = _two_stage([dish], sun=Sun("p", 4.65, (0.0, 0.0, 3.0), point_source=True), n=500)
    S["sun_oblique"] = _two_stage([dish], sun=Sun("p", 4.65, (30.0, -20.0, 60.0)))
    pill = OpticSet("pill", OpticFace("p", refl=0.9, slope=3.0, spec=1.0), OpticFace("p", refl=0.9, slope=3.0, spec=1.0))
    diff = OpticSet("diffuse", OpticFace("f", refl=0.8, slope=1.0, spec=0.0), OpticFace("f", refl=0.8))
    S["optics_pillbox"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="p",
                                              surface_params=(0.125, 0.125), origin=(0, 0, 0), aim=(0, 0, 1),
                                              interaction=2, optic="pill")], optics=[pill, TARGET])
    S["optics_diffuse"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="f", origin=(0, 0, 0),
                                              aim=(0, 0, 1), interaction=2, optic="diffuse")], optics=[diff, TARGET])
    ang = np.array([0.0, 200.0, 500.0, 900.0, 1400.0])
    tab = OpticSet("tab", OpticFace("g", refl=0.9, slope=1.0, refl_table=(ang, np.array([0.95, 0.9, 0.8, 0.6, 0.3]))),
                   OpticFace("g", refl=0.9))
    S["refl_table"] = _two_stage([Element(aperture="c", aperture_params=(4.0,), surface="p", surface_params=(0.125, 0.125),
                                          origin=(0, 0, 0), aim=(0, 0, 1), interaction=2, optic="tab")],
                                 optics=[tab, TARGET], sun=Sun("p", 4.65, (40.0, 0.0, 60.0)))
    # refraction through a glass slab, with a transmissivity table on one face
    glass = OpticSet("glass", OpticFace("g", trans=0.95, n_real=1.5,
                                        trans_table=(ang, np.array([0.97, 0.95, 0.9, 0.8, 0.5]))),
                     OpticFace("g", trans=0.95, n_real=1.0))
    slab = [Element(origin=(0, 0, 1.0), aim=(0, 0, 2.0), aperture="c", aperture_params=(4.0,), surface="f",
                    interaction=1, optic="glass"),
            Element(origin=(0, 0, 0.8), aim=(0, 0, 1.8), aperture="c", aperture_params=(4.0,), surface="s",
                    surface_params=(-0.05,), interaction=1, optic="glass")]
    floor = Element(origin=(0, 0, -3.0), aim=(0, 0, 0), aperture="r", aperture_params=(30, 30), surface="f",
                    interaction=2, optic="target")
    S["refraction"] = Scene(Sun("p", 4.65, (10.0, 5.0, 100.0)), [glass, TARGET],
                            [Stage(slab), Stage([floor])], raycount=3000, raymax=1_000_000)
    # stage flags
    S["virtual_stage"] = Scene(Sun("p", 4.65, (0.0, 0.0, 100.0)), [MIRROR, TARGET],
                               [Stage([Element(origin=(0, 0, 8), aim=(0, 0, 9), aperture="r", aperture_params=(6, 6),
                                               surface="f", interaction=2, optic="mirror")], virtual=True),
                                Stage([dish]), Stage([_target()])], raycount=3000, raymax=1_000_000)
    S["tracethrough"] = Scene(Sun("p", 4.65, (0.0, 0.0, 100.0)), [MIRROR, TARGET],
                              [Stage([dish]),
                               Stage([Element(origin=(0.7, 0, 2.0), aim=(0.7, 0, 0), aperture="c", aperture_params=(0.6,),
                                              surface="f", interaction=2, optic="mirror")], tracethrough=True),
                               Stage([_target()])], raycount=3000, raymax=1_000_000)
    S["no_multihit"] = _two_stage([dish, Element(origin=(0, 0, 1.2), aim=(0, 0, 0), aperture="c",
                                                 aperture_params=(1.0,), surface="s", surface_params=(0.3,),
                                                 interaction=2, optic="mirror")], multihit=False)
    S["multi_element"] = _two_stage([Element(origin=(x, y, 0), aim=(x * 0.1, y * 0.1, 5), aperture="r",
                                             aperture_params=(1.2, 1.2), surface="f", interaction=2, optic="mirror")
                                     for x in (-1.5, 0.0, 1.5) for y in (-1.5, 0.0, 1.5)] +
                                    [Element(origin=(0.4, 0.3, 2.0), aim=(0, 0, 0), aperture="c",
                                             aperture_params=(0.8,), surface="s", surface_params=(0.2,),
                                             interaction=2, optic="mirror")])
    return S
