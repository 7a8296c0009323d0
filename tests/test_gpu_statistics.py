"""Statistical-mode parity of the CUDA trace with the reference's own CPU trace.

The reference's random stream (one libstdc++ minstd_rand0 per context) and the device's
(per-ray Philox) differ, so results agree only within Monte-Carlo error.  The fixture
tests/golden/reference_stats.npz holds the reference's results, made by
tests/golden/make_stat_fixtures.py from the reference built from its own sources.

* Headline field (2,000 flat heliostats, Buie CSR 0.1 table sunshape, cylindrical
  receiver, 1e7 first-stage hits; the reference with exact culling): the 100 x 100
  receiver flux map (chi-square over the bins, and the share of bins beyond 3 sigma), the
  total intercept and the sun rays per hit (3 sigma), the per-heliostat first hits and
  deliveries (chi-square), in FP64 and in mixed precision.
* Samplers: the table sunshape 'd' (the device inverts the CDF of theta I(theta); the
  reference rejects in 2-D, errors.cpp:160-185) and the diffuse distribution 'f'
  (errors.cpp:187-190), through the radial histogram of a far target (chi-square).

A chi-square p-value below 1e-3 fails (a correct trace fails one such test in a
thousand runs).
"""
import os

import numpy as np
import pytest

from soltrace_b200 import scenes
from stat_scenes import (FIELD_FLUX, field_stat_scene, rate_z, sampler_scenes, target_radial_from_records,
                         two_sample_chi2)

pytestmark = pytest.mark.gpu

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_stats.npz")
P_MIN = 1e-3


@pytest.fixture(scope="module")
def ref_stats():
    return dict(np.load(FIX))


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
def test_field_flux_and_intercept_match_reference(product, ref_stats, prec):
    sc, hits, _ = field_stat_scene()
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
    r_hits, r_sun, r_abs = (int(x) for x in ref_stats["field_totals"])
    assert st["ray_hits"] == hits
    # sun rays per numbered hit and the receiver intercept, within 3 sigma
    z_sun = rate_z(hits, st["sun_rays"], r_hits, r_sun)
    z_int = rate_z(int(flux.sum()), hits, r_abs, r_hits)
    assert abs(z_sun) < 3, (st["sun_rays"], r_sun, z_sun)
    assert abs(z_int) < 3, (int(flux.sum()), r_abs, z_int)
    # the receiver map, bin by bin
    chi2, dof, p = two_sample_chi2(flux, hits, ref_stats["field_flux"], r_hits)
    assert p > P_MIN, (chi2, dof, p)
    a, b = flux.astype(float) / hits, ref_stats["field_flux"].astype(float) / r_hits
    sig = np.sqrt(flux / hits ** 2 + ref_stats["field_flux"] / r_hits ** 2)
    beyond = np.mean(np.abs(a - b) > 3 * np.maximum(sig, 1e-300))
    assert beyond <= 0.01, beyond  # 0.27 % expected
    # per-heliostat intercept: first hits and deliveries
    for mine, theirs in ((first, ref_stats["field_first"]), (delivered, ref_stats["field_delivered"])):
        chi2, dof, p = two_sample_chi2(np.asarray(mine, dtype=np.int64), hits, theirs, r_hits)
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
