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


# ------------------------------------------------------------------------------------
# Batched annual trace: beam-down tower
# ------------------------------------------------------------------------------------
BEAM_DOWN_HEIGHT = 120.0     # secondary vertex height (m)
BEAM_DOWN_ECC = 1.3          # hyperboloid eccentricity
BEAM_DOWN_DIAM = 20.0        # secondary aperture diameter (m)
LIP_RA, LIP_RS = 10.0, 0.5   # torus lip: annular and cross-section radius (m)
FOCUS_BELOW_RIM = 1.0        # upper focus this far below the secondary's rim plane (m)
GROUND_HALF = 32.0           # ground receiver half-width (m): holds the beam diverging from the lower focus
GROUND_MAP = (3, 1, 0, 64, 64, -GROUND_HALF, GROUND_HALF, -GROUND_HALF, GROUND_HALF, 1)  # 64 x 64, absorbed


def _hyperboloid_sag(R: float, kappa: float, r: float) -> float:
    """Height above the vertex of x^2 + y^2 + kappa z^2 - 2 R z = 0 at radius r (the root
    nearest the vertex)."""
    return (R - math.sqrt(R * R - kappa * r * r)) / kappa


def beam_down_geometry(height: float = BEAM_DOWN_HEIGHT, ecc: float = BEAM_DOWN_ECC):
    """(vertex curvature c, kappa, upper focus height, lower focus height) of the convex
    hyperboloid secondary.  SolTrace's 'o' surface is x^2 + y^2 + kappa z^2 - 2 z / c = 0
    (kappa = 1 - e^2); its foci lie R/(1+e) above and R/(e-1) below the vertex, R = 1/c.
    A ray aimed at the upper focus meets the mirror only if that focus lies inside the bowl,
    below the rim plane: rays from heliostats 1 km out rise about 1.2 m over the last 10 m,
    so R is chosen (by bisection) to put the upper focus FOCUS_BELOW_RIM under the rim.
    The lower focus is then ~91 m up, and the beam spreads from it to the ground receiver."""
    kappa = 1.0 - ecc * ecc
    r = BEAM_DOWN_DIAM / 2.0

    def gap(R):  # focus height above the vertex minus (rim height - FOCUS_BELOW_RIM)
        return R / (1.0 + ecc) - (_hyperboloid_sag(R, kappa, r) - FOCUS_BELOW_RIM)

    lo, hi = 0.5, 10.0 * r
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if (gap(lo) <= 0.0) == (gap(mid) <= 0.0):
            lo = mid
        else:
            hi = mid
    R = 0.5 * (lo + hi)
    return 1.0 / R, kappa, height + R / (1.0 + ecc), height - R / (ecc - 1.0)


def beam_down_scene(n_helio: int = 10000, raycount: int = 1_000_000, sun_xyz=None, r_min: float = 100.0,
                    r_max: float | None = None, slope: float = 1.5, csr: float = 0.1) -> Scene:
    """Beam-down tower: the heliostat field layout of field_scene scaled to n_helio heliostats
    (same density), a convex hyperboloid secondary (eccentricity 1.3, kappa = -0.69, 20 m
    aperture, vertex at 120 m, surface 'o' of quadricsurfaceclosedform.cpp:129-148) with an
    absorbing torus lip (surface 'd', annular radius 10 m, cross-section 0.5 m, aperture 'a'
    as input.cpp:349-355 requires) around its rim, and a flat 64 m x 64 m ground receiver
    under the lower focus (beam_down_geometry).  The secondary's stage is single-hit: the 'o'
    surface equation also holds on the hyperboloid's second sheet, 25 m under the vertex and
    inside the circular aperture, which rays reflected toward the lower focus would otherwise
    meet.  The heliostats are aimed at the upper focus for `sun_xyz` (default: 45 deg
    elevation, south); st_b200_sim_run_batch re-aims them per sun position with that focus
    as its tracking target (beam_down_target)."""
    c, kappa, f1, _ = beam_down_geometry()
    if r_max is None:  # the density of the 2,000-heliostat field over 100-1000 m
        r_max = math.sqrt(n_helio / 2000.0 * (1000.0 ** 2 - r_min ** 2) + r_min ** 2)
    xy = field_layout(n_helio, r_min=r_min, r_max=r_max)
    s = _unit(sun_xyz) if sun_xyz is not None else sun_vector(45.0, 180.0)
    target = np.array([0.0, 0.0, f1])
    helios = []
    for (x, y) in xy:
        pos = np.array([x, y, 5.0])
        t = target - pos
        n = s + t / math.sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2])
        nn = math.sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])
        helios.append(Element(origin=tuple(pos), aim=tuple(pos + 100.0 * (n / nn)), aperture="r",
                              aperture_params=(10.0, 10.0), surface="f", interaction=2, optic="helio"))
    h = BEAM_DOWN_HEIGHT
    rim = beam_down_rim_height()
    secondary = Element(origin=(0.0, 0.0, h), aim=(0.0, 0.0, h + 100.0), aperture="c", aperture_params=(BEAM_DOWN_DIAM,),
                        surface="o", surface_params=(c, kappa), interaction=2, optic="secondary")
    lip = Element(origin=(0.0, 0.0, rim - LIP_RS), aim=(0.0, 0.0, rim + 100.0), aperture="a",
                  aperture_params=(0.0, 0.0, 360.0), surface="d", surface_params=(LIP_RA, LIP_RS), interaction=2,
                  optic="lip")
    ground = Element(origin=(0.0, 0.0, 0.0), aim=(0.0, 0.0, 100.0), aperture="r",
                     aperture_params=(2.0 * GROUND_HALF, 2.0 * GROUND_HALF),
                     surface="f", interaction=2, optic="receiver")
    optics = [OpticSet("helio", OpticFace("g", refl=0.9, slope=slope), OpticFace("g", refl=0.9, slope=slope)),
              OpticSet("secondary", OpticFace("g", refl=0.95, slope=0.5), OpticFace("g", refl=0.95, slope=0.5)),
              OpticSet("lip", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0)),
              OpticSet("receiver", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0))]
    t_, inten = buie_csr_table(csr)
    sun = Sun("d", 0.0, tuple(1.0e4 * s), table=(t_, inten))
    return Scene(sun, optics, [Stage(helios), Stage([secondary, lip], multihit=False), Stage([ground])],
                 raycount=raycount, raymax=2_000_000_000 - 1, dynamic_group=True, name="beam_down")


def beam_down_rim_height() -> float:
    """Height of the secondary's rim (r = 10 m)."""
    c, kappa, _, _ = beam_down_geometry()
    return BEAM_DOWN_HEIGHT + _hyperboloid_sag(1.0 / c, kappa, BEAM_DOWN_DIAM / 2.0)


def beam_down_target() -> np.ndarray:
    """The heliostats' aim point: the hyperboloid's upper focus."""
    return np.array([0.0, 0.0, beam_down_geometry()[2]])


def sun_position(lat: float, day: float, hour: float):
    """(elevation, azimuth from north) in degrees by the formula of coretrace/stapi.cpp:500-527."""
    d2r = math.pi / 180.0
    decl = math.degrees(math.asin(0.39795 * math.cos(0.98563 * d2r * (day - 173))))
    ha = 15.0 * (hour - 12.0)
    el = math.degrees(math.asin(math.sin(decl * d2r) * math.sin(lat * d2r) +
                                math.cos(decl * d2r) * math.cos(ha * d2r) * math.cos(lat * d2r)))
    az = math.degrees(math.acos((math.sin(d2r * decl) * math.cos(d2r * lat) -
                                 math.cos(d2r * decl) * math.sin(d2r * lat) * math.cos(d2r * ha)) /
                                math.cos(d2r * el) + 1e-10))
    if math.sin(ha * d2r) > 0.0:
        az = 360.0 - az
    return el, az


def annual_suns(n: int = 512, lat: float = 40.0, seed: int = 7, min_elevation: float = 5.0, rays_per_kw: float = 1e6):
    """n sun positions drawn uniformly over the daylight hours of a year at latitude `lat`
    (day and hour uniform, kept when the sun is above min_elevation), each with a DNI drawn
    uniform in 300-1000 W/m2 and a hit budget of rays_per_kw x DNI / 1000.
    Returns (sun_xyz (n, 3) at 1e4 m, hits (n,), dni (n,))."""
    rng = np.random.default_rng(seed)
    suns, dni = [], []
    while len(suns) < n:
        day, hour = rng.uniform(1.0, 366.0), rng.uniform(0.0, 24.0)
        el, az = sun_position(lat, day, hour)
        if el < min_elevation:
            continue
        suns.append(1.0e4 * sun_vector(el, az))
        dni.append(rng.uniform(300.0, 1000.0))
    dni = np.asarray(dni)
    return np.asarray(suns), np.maximum(1, (rays_per_kw * dni / 1000.0).astype(np.int64)), dni
