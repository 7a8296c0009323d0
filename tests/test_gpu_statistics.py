"""Statistical-mode parity of the CUDA trace with the reference's own CPU trace.

The reference's random stream (one libstdc++ minstd_rand0 per context) and the device's
(per-ray Philox) differ, so results agree only within Monte-Carlo error.  The fixture
tests/golden/reference_stats.npz holds the reference's results, made by
tests/golden/make_stat_fixtures.py from the reference built from its own sources, every
reference thread on its own stretch of the generator's cycle.

* The headline field (2,000 flat heliostats, cylindrical receiver; the reference with exact
  culling), traced by the device to 1e7 first-stage hits, under the headline Buie CSR 0.1
  table sunshape and under a 2.73 mrad Gaussian sun: the 100 x 100 receiver flux map by
  chi-square and by the share of bins beyond 3 sigma, the total intercept and the sun rays
  per hit within 3 sigma, the per-heliostat first hits and deliveries by chi-square; FP64
  and mixed precision.  The reference's side holds 4e6 hits for the Buie sun (the most its
  generator's cycle holds without repeating random numbers: stat_scenes.REFERENCE_HITS) and
  1e7 for the Gaussian sun.
* Samplers: the table sunshape against the distribution the table defines and against the
  reference, and the diffuse distribution 'f' (errors.cpp:187-190) against the reference.

A chi-square p-value below 1e-3 fails (a correct trace fails one such test in a thousand).
"""
import os

import numpy as np
import pytest

from soltrace_b200 import scenes
from stat_scenes import (FIELD_FLUX, field_stat_scene, one_sample_chi2, rate_z, sampler_scenes, sun_theta_scene,
                         target_radial_from_records, theta_exact, theta_histogram, two_sample_chi2)

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_stats.npz")
P_MIN = 1e-3


@pytest.fixture(scope="module")
def ref_stats():
    return dict(np.load(FIX))


def _field_run(product, sun, prec):
    sc, hits, _ = field_stat_scene(sun)
    n_el = len(sc.stages[0].elements)
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_set_precision(ctx, prec)
        product.st_b200_set_records(ctx, 0)
        product.st_b200_add_flux_map(ctx, *FIELD_FLUX)
        assert product.run(ctx, 41) >= 0, product.messages(ctx)
        flux = product.flux(ctx, 0, FIELD_FLUX[3], FIELD_FLUX[4]).astype(np.int64)
        first, _, delivered = product.element_counts(ctx, 1, n_el)
        st = product.stats(ctx)
    finally:
        product.st_free_context(ctx)
    assert st["ray_hits"] == hits
    return hits, st, flux, np.asarray(first, dtype=np.int64), np.asarray(delivered, dtype=np.int64)


def _beyond_3_sigma(a, na, b, nb):
    pa, pb = a / na, b / nb
    sig = np.sqrt(a / na ** 2 + b / nb ** 2)
    m = (a + b) >= 10
    return float(np.mean(np.abs(pa - pb)[m] > 3 * sig[m]))


def _compare_totals(key, ref_stats, hits, st, flux, first):
    r_hits, r_sun, r_abs = (int(x) for x in ref_stats[f"{key}_totals"])
    z_sun = rate_z(hits, st["sun_rays"], r_hits, r_sun)
    z_int = rate_z(int(flux.sum()), hits, r_abs, r_hits)
    assert abs(z_sun) < 3, (st["sun_rays"], r_sun, z_sun)
    assert abs(z_int) < 3, (int(flux.sum()), r_abs, z_int)
    # first heliostat hit by each numbered ray: the sun-box sampling and the first stage only
    chi2, dof, p = two_sample_chi2(first, hits, ref_stats[f"{key}_first"], r_hits)
    assert p > P_MIN, ("first hits", chi2, dof, p)
    return r_hits


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("sun", ["buie", "gauss"])
def test_field_matches_reference(product, ref_stats, sun, prec):
    key = "field" if sun == "buie" else "field_gauss"
    hits, st, flux, first, delivered = _field_run(product, sun, prec)
    r_hits = _compare_totals(key, ref_stats, hits, st, flux, first)
    chi2, dof, p = two_sample_chi2(flux, hits, ref_stats[f"{key}_flux"], r_hits)
    assert p > P_MIN, ("flux map", chi2, dof, p)
    assert _beyond_3_sigma(flux, hits, ref_stats[f"{key}_flux"], r_hits) <= 0.01  # 0.27 % expected
    chi2, dof, p = two_sample_chi2(delivered, hits, ref_stats[f"{key}_delivered"], r_hits)
    assert p > P_MIN, ("deliveries", chi2, dof, p)


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
def test_table_sampler_draws_exact_distribution(product, prec):
    """The device's table-sunshape sampler against the angle distribution the table defines,
    p(theta) ~ theta I(theta) (errors.cpp:160-185), over 4e6 draws."""
    hits = 4_000_000
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sun_theta_scene(hits))
        product.st_b200_set_precision(ctx, prec)
        assert product.run(ctx, 19) > 0, product.messages(ctx)
        h = theta_histogram(product.records(ctx))
    finally:
        product.st_free_context(ctx)
    assert h.sum() == hits
    chi2, dof, p = one_sample_chi2(h, theta_exact())
    assert p > P_MIN, (chi2, dof, p)


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", ["sun_table", "diffuse"])
def test_samplers_match_reference(product, ref_stats, name, prec):
    sc, hits, _, rmax, nbins = sampler_scenes()[name]
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_set_precision(ctx, prec)
        assert product.run(ctx, 17) > 0, product.messages(ctx)
        h, on_target = target_radial_from_records(product.records(ctx), rmax, nbins)
    finally:
        product.st_free_context(ctx)
    r_hits, r_on = (int(x) for x in ref_stats[f"{name}_totals"])
    assert abs(rate_z(on_target, hits, r_on, r_hits)) < 3
    chi2, dof, p = two_sample_chi2(h, hits, ref_stats[f"{name}_radial"], r_hits)
    assert p > P_MIN, (name, chi2, dof, p)
