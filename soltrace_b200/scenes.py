"""Scene descriptions and the benchmark scenes, pushed into any library that
exports the stapi.h setters.

A `Scene` mirrors what a SolTrace front end (pysoltrace, the strace .stinput
reader, the GUI) sends through the C API: one sun, named optical property
sets, stages with elements, and the simulation parameters of st_sim_params /
st_sim_errors.  `push()` replays it with the same call order pysoltrace uses
(app/deploy/api/pysoltrace.py:392-451 optics, 514-540 sun, 1292-1319 stages,
735-777 elements): aperture before surface parameters, because the surface
translation depends on the aperture (coretrace/input.cpp:288-366).

The benchmark scenes are synthetic stand-ins built from their stated
dimensions; the sunshape of the field scene is the Buie et al. (2003) CSR model
evaluated on a 50-point table.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .capi import StApi, dptr


@dataclass
class OpticFace:
    dist: str = "g"
    refl: float = 0.0
    trans: float = 0.0
    slope: float = 0.0      # mrad
    spec: float = 0.0       # mrad
    n_real: float = 1.0
    n_imag: float = 0.0
    refl_table: tuple | None = None    # (angles mrad, values)
    trans_table: tuple | None = None


@dataclass
class OpticSet:
    name: str
    front: OpticFace = field(default_factory=OpticFace)
    back: OpticFace = field(default_factory=OpticFace)


@dataclass
class Element:
    origin: tuple = (0.0, 0.0, 0.0)
    aim: tuple = (0.0, 0.0, 1.0)
    zrot: float = 0.0
    aperture: str = "c"
    aperture_params: tuple = (1.0,)
    surface: str = "f"
    surface_params: tuple = ()
    surface_file: str | None = None
    interaction: int = 2
    optic: str = ""
    enabled: bool = True


@dataclass
class Stage:
    elements: list
    origin: tuple = (0.0, 0.0, 0.0)
    aim: tuple = (0.0, 0.0, 1.0)
    zrot: float = 0.0
    virtual: bool = False
    multihit: bool = True
    tracethrough: bool = False


@dataclass
class Sun:
    shape: str = "p"
    sigma: float = 4.65
    xyz: tuple = (0.0, 0.0, 100.0)
    point_source: bool = False
    table: tuple | None = None   # (angles mrad, intensities)


@dataclass
class Scene:
    sun: Sun
    optics: list
    stages: list
    raycount: int = 10000
    raymax: int = 10_000_000
    dynamic_group: bool = False
    sunshape_errors: bool = True
    optical_errors: bool = True
    name: str = "scene"

    def n_elements(self) -> int:
        return sum(len(s.elements) for s in self.stages)


def _pad8(v) -> np.ndarray:
    a = np.zeros(8)
    a[: len(v)] = v
    return a


def _face_args(f: OpticFace):
    keep = []

    def arr(x):
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
        keep.append(a)
        return dptr(a)

    grating = arr(np.zeros(4))
    rt = f.refl_table
    tt = f.trans_table
    args = (f.dist.encode()[:1], 1, 0, 0, f.n_real, f.n_imag, f.refl, f.trans, grating, f.slope, f.spec,
            1 if rt else 0, len(rt[0]) if rt else 0, arr(rt[0]) if rt else arr([0.0]), arr(rt[1]) if rt else arr([0.0]),
            1 if tt else 0, len(tt[0]) if tt else 0, arr(tt[0]) if tt else arr([0.0]), arr(tt[1]) if tt else arr([0.0]))
    return args, keep


def push_optic(api: StApi, ctx, idx: int, o: OpticSet) -> None:
    """Set both faces of optic `idx` (st_optic front, then back)."""
    for fb, face in ((1, o.front), (2, o.back)):
        args, keep = _face_args(face)
        rc = api.st_optic(ctx, idx, fb, *args)
        del keep
        if rc is not None and rc < 0:
            raise RuntimeError(f"st_optic failed ({rc}): {api.messages(ctx)}")


def push(api: StApi, ctx, sc: Scene) -> None:
    """Send the scene through the C API setters; raises on any setter failure."""

    def ok(rc, what):
        if rc is not None and rc < 0:
            raise RuntimeError(f"{what} failed ({rc}): {api.messages(ctx)}")

    for o in sc.optics:
        idx = api.st_add_optic(ctx, o.name.encode())
        push_optic(api, ctx, idx, o)
    ok(api.st_sun(ctx, int(sc.sun.point_source), sc.sun.shape.encode()[:1], sc.sun.sigma), "st_sun")
    ok(api.st_sun_xyz(ctx, *map(float, sc.sun.xyz)), "st_sun_xyz")
    if sc.sun.table is not None:
        ang = np.ascontiguousarray(sc.sun.table[0], dtype=np.float64)
        inten = np.ascontiguousarray(sc.sun.table[1], dtype=np.float64)
        ok(api.st_sun_userdata(ctx, len(ang), dptr(ang), dptr(inten)), "st_sun_userdata")
    for si, st in enumerate(sc.stages):
        api.st_add_stage(ctx)
        ok(api.st_stage_xyz(ctx, si, *map(float, st.origin)), "st_stage_xyz")
        ok(api.st_stage_aim(ctx, si, *map(float, st.aim)), "st_stage_aim")
        ok(api.st_stage_zrot(ctx, si, float(st.zrot)), "st_stage_zrot")
        ok(api.st_stage_flags(ctx, si, int(st.virtual), int(st.multihit), int(st.tracethrough)), "st_stage_flags")
        if st.elements:
            ok(api.st_add_elements(ctx, si, len(st.elements)), "st_add_elements")
        for ei, e in enumerate(st.elements):
            ok(api.st_element_enabled(ctx, si, ei, int(e.enabled)), "enabled")
            ok(api.st_element_xyz(ctx, si, ei, *map(float, e.origin)), "xyz")
            ok(api.st_element_aim(ctx, si, ei, *map(float, e.aim)), "aim")
            ok(api.st_element_zrot(ctx, si, ei, float(e.zrot)), "zrot")
            ok(api.st_element_aperture(ctx, si, ei, e.aperture.encode()[:1]), "aperture")
            ap = _pad8(e.aperture_params)
            ok(api.st_element_aperture_params(ctx, si, ei, dptr(ap)), "aperture params")
            ok(api.st_element_surface(ctx, si, ei, e.surface.encode()[:1]), "surface")
            if e.surface_file:
                ok(api.st_element_surface_file(ctx, si, ei, e.surface_file.encode()), "surface file")
            else:
                sp = _pad8(e.surface_params)
                ok(api.st_element_surface_params(ctx, si, ei, dptr(sp)), "surface params")
            ok(api.st_element_interaction(ctx, si, ei, int(e.interaction)), "interaction")
            ok(api.st_element_optic(ctx, si, ei, e.optic.encode()), "optic")
    ok(api.st_sim_params(ctx, int(sc.raycount), int(sc.raymax), int(sc.dynamic_group)), "st_sim_params")
    ok(api.st_sim_errors(ctx, int(sc.sunshape_errors), int(sc.optical_errors)), "st_sim_errors")


# ------------------------------------------------------------------------------------
# Benchmark scenes
# ------------------------------------------------------------------------------------
def dish_scene(raycount: int = 1_000_000, focal: float = 5.0, diameter: float = 10.0,
               absorber_d: float = 0.5) -> Scene:
    """Parabolic dish + flat circular absorber (pillbox sun 4.65 mrad along -z)."""
    c = 1.0 / (2.0 * focal)
    optics = [
        OpticSet("mirror", OpticFace("g", refl=0.9, slope=2.0, spec=0.5), OpticFace("g", refl=0.9, slope=2.0, spec=0.5)),
        OpticSet("absorber", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0)),
    ]
    dish = Element(origin=(0, 0, 0), aim=(0, 0, 1), aperture="c", aperture_params=(diameter,),
                   surface="p", surface_params=(c, c), interaction=2, optic="mirror")
    absorber = Element(origin=(0, 0, focal), aim=(0, 0, 0), aperture="c", aperture_params=(absorber_d,),
                       surface="f", interaction=2, optic="absorber")
    return Scene(Sun("p", 4.65, (0.0, 0.0, 100.0)), optics,
                 [Stage([dish]), Stage([absorber])], raycount=raycount, raymax=100 * raycount + 1000,
                 name="dish")


def trough_scene(raycount: int = 10_000_000, focal: float = 1.71, width: float = 5.77, length: float = 12.0,
                 elevation_deg: float = 60.0) -> Scene:
    """Parabolic trough with a glass envelope and an absorber tube.

    Stage 1 is the single-axis parabolic reflector ('p', Cy = 0, aperture 'l').
    Stage 2 is the outer wall of the glass envelope (r = 62.5 mm), traced once per
    ray (no multi-hit), so rays enter the glass.  Stage 3 holds the inner wall
    (r = 59.5 mm) and the absorber tube (r = 35 mm) with multi-hit on, so rays
    cross into the annulus and reach the absorber.  All tubes are centred on the
    focal line z = f.  The cylinders' gradient points at their axis, so a ray
    arriving from outside meets the 'back' face: the back face carries the
    outside medium's index (coretrace/input.cpp:272-275 cross-wires the rest).
    """
    c = 1.0 / (2.0 * focal)
    r_out, r_in, r_abs = 0.0625, 0.0595, 0.035
    el = math.radians(elevation_deg)
    optics = [
        OpticSet("mirror", OpticFace("g", refl=0.94, slope=2.5, spec=0.0), OpticFace("g", refl=0.94, slope=2.5)),
        OpticSet("glass_out", OpticFace("g", trans=0.965, n_real=1.52), OpticFace("g", trans=0.965, n_real=1.0)),
        OpticSet("glass_in", OpticFace("g", trans=1.0, n_real=1.0), OpticFace("g", trans=1.0, n_real=1.52)),
        OpticSet("absorber", OpticFace("g", refl=0.05), OpticFace("g", refl=0.05)),
    ]
    refl = Element(origin=(0, 0, 0), aim=(0, 0, 1), aperture="l", aperture_params=(-width / 2, width / 2, length),
                   surface="p", surface_params=(c, 0.0), interaction=2, optic="mirror")

    def tube(r, optic, interaction):
        z0 = focal - r
        return Element(origin=(0, 0, z0), aim=(0, 0, z0 + 1.0), aperture="l", aperture_params=(0.0, 0.0, length),
                       surface="t", surface_params=(1.0 / r,), interaction=interaction, optic=optic)

    stages = [Stage([refl]),
              Stage([tube(r_out, "glass_out", 1)], multihit=False),
              Stage([tube(r_in, "glass_in", 1), tube(r_abs, "absorber", 2)])]
    sun = Sun("g", 2.73, (0.0, 100.0 * math.cos(el), 100.0 * math.sin(el)))
    return Scene(sun, optics, stages, raycount=raycount, raymax=100 * raycount + 1000, name="trough")


def buie_csr_table(csr: float, n: int = 50, max_mrad: float = 30.0):
    """Buie, Monger & Dey (2003) sunshape: cos(0.326 t)/cos(0.308 t) inside the
    4.65 mrad solar disc, exp(kappa) t^gamma in the aureole, with
    kappa = 0.9 ln(13.5 chi) chi^-0.3 and gamma = 2.2 ln(0.52 chi) chi^0.43 - 0.1."""
    t = np.linspace(0.0, max_mrad, n)
    kappa = 0.9 * math.log(13.5 * csr) * csr ** -0.3
    gamma = 2.2 * math.log(0.52 * csr) * csr ** 0.43 - 0.1
    disc = np.cos(0.326 * t) / np.cos(0.308 * t)
    with np.errstate(divide="ignore"):
        aureole = np.exp(kappa) * np.power(np.maximum(t, 1e-9), gamma)
    inten = np.where(t <= 4.65, disc, aureole)
    return t, inten / inten.max()


def field_layout(n_helio: int = 2000, r_min: float = 100.0, r_max: float = 1000.0, width: float = 10.0,
                 spacing: float = 1.6) -> np.ndarray:
    """Radial-staggered layout north of the tower (azimuth within +-90 deg of +y).
    Rows are evenly spaced in radius; each row holds as many heliostats as fit
    at `spacing` widths apart, alternate rows shifted by half a slot; the first
    n_helio positions in row order are kept."""
    pts = []
    n_rows = 2
    while True:
        radii = np.linspace(r_min, r_max, n_rows)
        cap = sum(int(math.pi * r / (spacing * width)) for r in radii)
        if cap >= n_helio:
            break
        n_rows += 1
    for k, r in enumerate(radii):
        m = int(math.pi * r / (spacing * width))
        dphi = math.pi / m
        off = 0.5 * dphi if k % 2 else 0.0
        for j in range(m):
            az = -math.pi / 2 + (j + 0.5) * dphi + off
            if az > math.pi / 2:
                continue
            pts.append((r * math.sin(az), r * math.cos(az)))
    pts = np.asarray(pts[:n_helio])
    return pts


def _unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def sun_vector(elevation_deg: float, azimuth_deg: float) -> np.ndarray:
    """Unit vector toward the sun; x = east, y = north, z = up, azimuth from north."""
    el, az = math.radians(elevation_deg), math.radians(azimuth_deg)
    return np.array([math.cos(el) * math.sin(az), math.cos(el) * math.cos(az), math.sin(el)])


def field_scene(n_helio: int = 2000, raycount: int = 100_000_000, elevation_deg: float = 45.0,
                azimuth_deg: float = 180.0, tower_h: float = 150.0, rec_d: float = 8.0, rec_h: float = 10.0,
                aim_sigma: float = 0.3, slope: float = 1.5, csr: float = 0.1, seed: int = 3,
                dynamic_group: bool = True) -> Scene:
    """Central receiver: flat 10x10 m heliostats on a radial-staggered field north of
    the tower, each aimed by the bisector rule at the receiver centre plus a
    per-heliostat Gaussian aim offset; external cylindrical receiver whose
    element axis is vertical (aimed horizontally, as in the reference samples)."""
    rng = np.random.default_rng(seed)
    xy = field_layout(n_helio)
    s = sun_vector(elevation_deg, azimuth_deg)
    target = np.array([0.0, 0.0, tower_h])
    helios = []
    z_h = 5.0  # pivot height
    for (x, y) in xy:
        pos = np.array([x, y, z_h])
        aimpt = target + rng.normal(0.0, aim_sigma, 3)
        n = _unit(s + _unit(aimpt - pos))
        helios.append(Element(origin=tuple(pos), aim=tuple(pos + 100.0 * n), zrot=0.0, aperture="r",
                              aperture_params=(10.0, 10.0), surface="f", interaction=2, optic="helio"))
    r = rec_d / 2.0
    rec = Element(origin=(0.0, r, tower_h), aim=(0.0, r - 1.0, tower_h), aperture="l",
                  aperture_params=(0.0, 0.0, rec_h), surface="t", surface_params=(1.0 / r,),
                  interaction=2, optic="receiver")
    optics = [OpticSet("helio", OpticFace("g", refl=0.9, slope=slope, spec=0.0),
                       OpticFace("g", refl=0.9, slope=slope, spec=0.0)),
              OpticSet("receiver", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0))]
    t, inten = buie_csr_table(csr)
    sun = Sun("d", 0.0, tuple(1.0e4 * s), table=(t, inten))
    return Scene(sun, optics, [Stage(helios), Stage([rec])], raycount=raycount,
                 raymax=max(2_000_000_000 - 1, 0) if raycount > 10_000_000 else 200 * raycount + 10_000,
                 dynamic_group=dynamic_group, name="field")
