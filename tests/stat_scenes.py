"""Scenes and binning rules of the statistical parity tests.

Used by tests/golden/make_stat_fixtures.py (on the reference's records) and by the
statistical tests (on the CUDA trace's device maps and records, and on the oracle's).
The binning of the receiver map restates pysoltrace's cylinder flux map
(app/deploy/api/pysoltrace.py:1896-1942): element-local position, angle
atan2(x, z - r) + pi over [0, 2 pi) by axial y over [-H/2, H/2), absorbed rays only.
"""
from __future__ import annotations

import math

import numpy as np
from scipy import stats as sps

from soltrace_b200 import scenes
from soltrace_b200.scenes import Element, OpticFace, OpticSet, Scene, Stage, Sun

# receiver map of the heliostat field: stage 2, element 1, pysoltrace cylinder rule (kind 1),
# 100 angle x 100 axial bins, radius 4 m, axial [-5, 5] m, absorbed rays only
FIELD_FLUX = (2, 1, 1, 100, 100, 0.0, 4.0, -5.0, 5.0, 1)
FIELD_HELIOSTATS = 2000
FIELD_HITS = 10_000_000
FIELD_SEED = 3


def field_stat_scene(sun: str = "buie"):
    """The headline field (2,000 flat heliostats, 8 m x 10 m receiver) with exact culling on
    the reference's side (include_dynamic_group = 0); sun "buie": the headline Buie CSR 0.1
    table sunshape; "gauss": a Gaussian sunshape of sigma 2.73 mrad instead (whose sampler the
    reference draws without the table sampler's bias, see sun_theta_scene)."""
    import dataclasses
    sc = scenes.field_scene(FIELD_HELIOSTATS, FIELD_HITS, dynamic_group=False)
    if sun == "gauss":
        sc = dataclasses.replace(sc, sun=dataclasses.replace(sc.sun, shape="g", sigma=2.73, table=None))
    return sc, FIELD_HITS, FIELD_SEED


# The reference's generator has a single cycle of 2^31 - 2 states, which all its threads share.
# Its table-sunshape sampler (2-D rejection, about 2 % accepted) takes about 290 generator calls
# per sun angle, so the Buie-table field costs about 330 calls per first-stage hit and one cycle
# holds only about 6.5e6 hits: a longer reference run repeats its random numbers and its
# Monte-Carlo error stops shrinking.  The reference's fixtures therefore stay within the cycle:
# REFERENCE_HITS per configuration, each thread on its own stretch (spaced_seeds).
REFERENCE_CYCLE = 2 ** 31 - 2
REFERENCE_HITS = {"buie": 4_000_000, "gauss": 10_000_000}


def spaced_seeds(n: int, offset: int = 999):
    """Seeds for n reference threads whose random streams never overlap: the reference's
    generator is libstdc++'s minstd_rand0 (x <- 16807 x mod 2^31-1, seeded with x0 = seed),
    so seeding thread i with 16807^(i (2^31-2)/n + offset) starts it i/n of the way around
    the generator's cycle, and each thread owns (2^31-2)/n consecutive states."""
    M = 2 ** 31 - 1
    return [pow(16807, i * ((M - 1) // n) + offset, M) for i in range(n)]


# sun-angle sampler: a 0.2 mm flat mirror under the Buie CSR 0.1 table sunshape reflecting onto
# a target 500 m above it: a ray sampled at sun angle theta lands at radius 500 tan(theta)
THETA_HEIGHT, THETA_BINS, THETA_MAX = 500.0, 120, 30.0


def sun_theta_scene(hits: int):
    t, inten = scenes.buie_csr_table(0.1)
    sun = Sun("d", 0.0, (0.0, 0.0, 100.0), table=(t, inten))
    mirror = Element(origin=(0, 0, 0), aim=(0, 0, 1), aperture="c", aperture_params=(0.0002,), surface="f",
                     interaction=2, optic="mirror")
    target = Element(origin=(0, 0, THETA_HEIGHT), aim=(0, 0, 0), aperture="c", aperture_params=(40.0,), surface="f",
                     interaction=2, optic="target")
    optics = [OpticSet("mirror", OpticFace("g", refl=1.0), OpticFace("g", refl=1.0)),
              OpticSet("target", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0))]
    return Scene(sun, optics, [Stage([mirror]), Stage([target])], raycount=hits, raymax=100 * hits + 1000)


def theta_histogram(rec: dict) -> np.ndarray:
    """Histogram of the sampled sun angles (mrad, THETA_BINS bins over [0, THETA_MAX]) from the
    target hits of sun_theta_scene."""
    sel = rec["stage"] == 2
    r = np.hypot(rec["x"][sel], rec["y"][sel])
    return np.histogram(np.arctan(r / THETA_HEIGHT) * 1000.0, bins=THETA_BINS, range=(0.0, THETA_MAX))[0].astype(np.int64)


def theta_exact() -> np.ndarray:
    """Bin probabilities of the sun angle the table sunshape defines: p(theta) ~ theta I(theta)
    on [0, 30] mrad with I linearly interpolated on the table (errors.cpp:160-185: a point drawn
    uniformly in the square of half-side MaxAngle, kept with probability I(theta)/I_max inside
    the circle of radius MaxAngle), integrated numerically."""
    t, inten = scenes.buie_csr_table(0.1)
    th = np.linspace(0.0, THETA_MAX, 3_000_001)
    pdf = th * np.interp(th, t, inten)
    cdf = np.concatenate([[0.0], np.cumsum((pdf[1:] + pdf[:-1]) / 2.0 * np.diff(th))])
    cdf /= cdf[-1]
    return np.diff(np.interp(np.linspace(0.0, THETA_MAX, THETA_BINS + 1), th, cdf))


def one_sample_chi2(h: np.ndarray, p: np.ndarray, min_expected: float = 5.0):
    """Goodness of fit of histogram h to bin probabilities p: (chi2, dof, p-value)."""
    n = h.sum()
    e = n * p
    k = e > min_expected
    chi2 = float(((h[k] - e[k]) ** 2 / e[k]).sum())
    dof = int(k.sum()) - 1
    return chi2, dof, float(sps.chi2.sf(chi2, dof))


def _mirror_target(sun: Sun, optic: OpticFace, height: float, target_d: float, hits: int) -> Scene:
    mirror = Element(origin=(0, 0, 0), aim=(0, 0, 1), aperture="c", aperture_params=(0.1,), surface="f",
                     interaction=2, optic="mirror")
    target = Element(origin=(0, 0, height), aim=(0, 0, 0), aperture="c", aperture_params=(target_d,), surface="f",
                     interaction=2, optic="target")
    optics = [OpticSet("mirror", optic, optic),
              OpticSet("target", OpticFace("g", refl=0.0), OpticFace("g", refl=0.0))]
    return Scene(sun, optics, [Stage([mirror]), Stage([target])], raycount=hits, raymax=100 * hits + 1000)


def sampler_scenes() -> dict:
    """name -> (scene, hits, seed, histogram radius, bins).

    sun_table: the field's Buie CSR 0.1 table sunshape on a perfect flat mirror (no optical
      errors) reflecting onto a target 500 m above it; a ray sampled at sun angle theta lands
      at radius 500 tan(theta) (+- the 5 cm mirror), so the radial histogram is the sampled
      angle distribution up to the table's 30 mrad.
    diffuse: the diffuse distribution 'f' (angle asin(sqrt(u)) about the normal) on the same
      mirror under a 0.1 mrad pillbox sun, onto a 60 m target 10 m above it (angles to 71.6
      degrees)."""
    t, inten = scenes.buie_csr_table(0.1)
    table_sun = Sun("d", 0.0, (0.0, 0.0, 100.0), table=(t, inten))
    perfect = OpticFace("g", refl=1.0, slope=0.0, spec=0.0)
    diffuse = OpticFace("f", refl=1.0, slope=0.0, spec=1.0)
    return {
        "sun_table": (_mirror_target(table_sun, perfect, 500.0, 40.0, 1_000_000), 1_000_000, 5, 16.0, 64),
        "diffuse": (_mirror_target(Sun("p", 0.1, (0.0, 0.0, 100.0)), diffuse, 10.0, 60.0, 1_000_000), 1_000_000, 6,
                    30.0, 60),
    }


def _element_frame(api, el: Element):
    """Rotation (reference -> local) and origin of an element, from the library's own
    transform utilities (st_calc_euler_angles, st_calc_transform_matrices)."""
    from soltrace_b200.capi import dptr
    o = np.ascontiguousarray(el.origin, dtype=np.float64)
    a = np.ascontiguousarray(el.aim, dtype=np.float64)
    eu = np.zeros(3)
    api.st_calc_euler_angles(dptr(o), dptr(a), float(el.zrot), dptr(eu))
    r2l = np.zeros((3, 3))
    l2r = np.zeros((3, 3))
    api.st_calc_transform_matrices(dptr(eu), dptr(r2l), dptr(l2r))
    return r2l, o


def receiver_flux_from_records(api, sc: Scene, rec: dict) -> np.ndarray:
    """FIELD_FLUX bins ([iy][ix]) of the absorbed receiver records (stage 2, element -1)."""
    stage, elem, kind, nx, ny, _, radius, y0, y1, _ = FIELD_FLUX
    sel = (rec["stage"] == stage) & (rec["element"] == -elem)
    p = np.column_stack([rec["x"][sel], rec["y"][sel], rec["z"][sel]])
    r2l, o = _element_frame(api, sc.stages[stage - 1].elements[elem - 1])
    loc = (p - o) @ r2l.T
    ang = np.arctan2(loc[:, 0], loc[:, 2] - radius) + math.pi
    ix = np.floor(ang * nx / (2 * math.pi)).astype(np.int64)
    iy = np.floor((loc[:, 1] - y0) / (y1 - y0) * ny).astype(np.int64)
    ok = (ix >= 0) & (ix < nx) & (iy >= 0) & (iy < ny)
    out = np.zeros((ny, nx), dtype=np.int64)
    np.add.at(out, (iy[ok], ix[ok]), 1)
    return out


def per_heliostat_from_records(rec: dict, n_el: int):
    """(first hits, deliveries) per heliostat: a ray's first heliostat is its first stage-1
    record; it is delivered when it has an absorbed stage-2 record."""
    s1 = rec["stage"] == 1
    rn1, el1 = rec["raynum"][s1], np.abs(rec["element"][s1])
    # readback keeps each ray's hits of a stage in order, so the first occurrence is the first hit
    order = np.argsort(rn1, kind="stable")
    rn1, el1 = rn1[order], el1[order]
    head = np.r_[True, rn1[1:] != rn1[:-1]]
    first_ray, first_el = rn1[head], el1[head]
    first = np.bincount(first_el - 1, minlength=n_el)
    absorbed_rays = np.unique(rec["raynum"][(rec["stage"] == 2) & (rec["element"] < 0)])
    got = np.isin(first_ray, absorbed_rays)
    delivered = np.bincount(first_el[got] - 1, minlength=n_el)
    return first.astype(np.int64), delivered.astype(np.int64)


def target_radial_from_records(rec: dict, rmax: float, nbins: int):
    """Radial histogram of the absorbed target hits (stage 2) over [0, rmax), and their count."""
    sel = (rec["stage"] == 2) & (rec["element"] < 0)
    r = np.hypot(rec["x"][sel], rec["y"][sel])
    h, _ = np.histogram(r, bins=nbins, range=(0.0, rmax))
    return h.astype(np.int64), int(sel.sum())


def two_sample_chi2(a: np.ndarray, na: float, b: np.ndarray, nb: float, min_count: int = 10):
    """Chi-square test that binned counts a (out of na trials) and b (out of nb) come from the
    same per-trial bin probabilities.  Bins with fewer than min_count events in both are
    pooled into one.  Returns (chi2, dof, p-value)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    small = (a + b) < min_count
    if small.any():
        a = np.r_[a[~small], a[small].sum()]
        b = np.r_[b[~small], b[small].sum()]
    keep = (a + b) > 0
    a, b = a[keep], b[keep]
    ka, kb = math.sqrt(nb / na), math.sqrt(na / nb)
    chi2 = float(np.sum((ka * a - kb * b) ** 2 / (a + b)))
    dof = len(a)
    return chi2, dof, float(sps.chi2.sf(chi2, dof))


def rate_z(ka: float, na: float, kb: float, nb: float) -> float:
    """z-score of the difference of two binomial rates ka/na and kb/nb."""
    pa, pb = ka / na, kb / nb
    p = (ka + kb) / (na + nb)
    s = math.sqrt(max(p * (1 - p), 1e-300) * (1 / na + 1 / nb))
    return (pa - pb) / s
