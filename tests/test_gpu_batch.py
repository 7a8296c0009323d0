"""Batched multi-sun runs (st_b200_sim_run_batch) against single runs.

Position k of a batch draws from the streams of seed + k, so it must give exactly what
st_sim_run(seed + k) gives on the same scene with sun k: the same SunRayCount, hits,
stage entries and intersection count, the same ground-receiver flux bins and the same
absorbed count on every element of every stage (all integer, so any ray traced
differently shows).  Checked on the beam-down scene (heliostat field, hyperboloid
secondary with a torus lip, ground receiver), for a fixed field and for a field that
tracks the sun (re-aimed per position), in FP64 and mixed precision.  The single runs
use the outgoing-beam lists for the heliostats' blocking searches and the batch does not,
so the equality also checks that both searches are exact.
"""
import numpy as np
import pytest

from soltrace_b200 import scenes

pytestmark = pytest.mark.gpu

N_HELIO = 1500
GM = scenes.GROUND_MAP


def _single(product, sc, sun_xyz, hits, seed, prec):
    import dataclasses
    sc = dataclasses.replace(sc, sun=dataclasses.replace(sc.sun, xyz=tuple(float(v) for v in sun_xyz)), raycount=int(hits))
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_set_precision(ctx, prec)
        product.st_b200_set_records(ctx, 0)
        product.st_b200_add_flux_map(ctx, *GM)
        assert product.run(ctx, seed) >= 0, product.messages(ctx)
        st = product.stats(ctx)
        flux = product.flux(ctx, 0, GM[3], GM[4])
        absorbed = [product.element_counts(ctx, s + 1, len(stg.elements))[1] for s, stg in enumerate(sc.stages)]
        box = product.sun_stats(ctx)
    finally:
        product.st_free_context(ctx)
    return st, flux, absorbed, box


def _compare(product, ctx, k, sc, ref):
    st, flux, absorbed, box = ref
    b = product.batch_stats(ctx, k)
    for key in ("sun_rays", "ray_hits", "ray_stage_units", "intersections"):
        assert b[key] == st[key], (k, key, b[key], st[key])
    assert b["stage_entries"][:3] == st["stage_entries"][:3]
    np.testing.assert_array_equal(product.batch_flux(ctx, 0, k, GM[3], GM[4]), flux)
    for s, stg in enumerate(sc.stages):
        np.testing.assert_array_equal(product.batch_absorbed(ctx, k, s + 1, len(stg.elements)), absorbed[s])
    xmin, xmax, ymin, ymax = product.batch_sun_box(ctx, k)
    assert (xmin, xmax, ymin, ymax) == (box["xmin"], box["xmax"], box["ymin"], box["ymax"])


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("tracking", [False, True], ids=["fixed", "tracking"])
def test_batch_positions_equal_single_runs(product, prec, tracking):
    suns, _, _ = scenes.annual_suns(3, seed=11)
    hits = [20000, 6000, 30000]
    seed = 40
    sc = scenes.beam_down_scene(N_HELIO, raycount=1000)
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_set_precision(ctx, prec)
        product.st_b200_add_flux_map(ctx, *GM)
        target = scenes.beam_down_target() if tracking else None
        assert product.run_batch(ctx, seed, suns, hits, target) == 1, product.messages(ctx)
        total = product.batch_stats(ctx, -1)
        assert total["ray_hits"] == sum(hits)
        for k in range(len(hits)):
            # with tracking, the single run's heliostats are aimed for sun k by the same rule
            sk = scenes.beam_down_scene(N_HELIO, raycount=1000, sun_xyz=suns[k]) if tracking else sc
            ref = _single(product, sk, suns[k], hits[k], seed + k, prec)
            # rays reach the secondary (and, when the field tracks the sun, the ground receiver)
            assert ref[0]["stage_entries"][1] > 0
            if tracking:
                assert ref[0]["stage_entries"][2] > 0
            _compare(product, ctx, k, sk, ref)
    finally:
        product.st_free_context(ctx)


def test_batch_zero_budget_and_repeat(product):
    """A position with no hits has SunRayCount 0; a second call on the same context gives
    the same results (the per-position state is reset)."""
    suns, _, _ = scenes.annual_suns(2, seed=3)
    sc = scenes.beam_down_scene(N_HELIO, raycount=1000)
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_add_flux_map(ctx, *GM)
        out = []
        for _ in range(2):
            assert product.run_batch(ctx, 9, suns, [0, 5000], scenes.beam_down_target()) == 1, product.messages(ctx)
            out.append((product.batch_stats(ctx, 0), product.batch_stats(ctx, 1),
                        product.batch_flux(ctx, 0, 1, GM[3], GM[4])))
        assert out[0][0]["sun_rays"] == 0 and out[0][0]["ray_hits"] == 0
        assert out[0][1]["ray_hits"] == 5000
        assert out[0][1]["sun_rays"] == out[1][1]["sun_rays"]
        np.testing.assert_array_equal(out[0][2], out[1][2])
    finally:
        product.st_free_context(ctx)


def test_batch_over_several_chunks_equals_separate_calls(product):
    """150 positions go to the device in three chunks, each staged (page-locked, on the host
    cores) while the device runs the previous one; every position must equal the same position
    run in a call of its own chunk-sized slice (seed offset so that it keeps its streams)."""
    n = 150
    suns, _, _ = scenes.annual_suns(n, seed=5)
    hits = [1500 + 37 * (k % 11) for k in range(n)]
    seed = 70
    sc = scenes.beam_down_scene(N_HELIO, raycount=1000)
    target = scenes.beam_down_target()

    def run(ctx, a, b):
        assert product.run_batch(ctx, seed + a, suns[a:b], hits[a:b], target) == 1, product.messages(ctx)
        return [(product.batch_stats(ctx, k), product.batch_flux(ctx, 0, k, GM[3], GM[4]),
                 product.batch_absorbed(ctx, k, 1, N_HELIO)) for k in range(b - a)]

    ctxs = []
    try:
        for _ in range(2):
            ctx = product.st_create_context()
            ctxs.append(ctx)
            scenes.push(product, ctx, sc)
            product.st_b200_set_precision(ctx, 1)
            product.st_b200_add_flux_map(ctx, *GM)
        whole = run(ctxs[0], 0, n)
        parts = run(ctxs[1], 0, 50) + run(ctxs[1], 50, 100) + run(ctxs[1], 100, n)
        for k in range(n):
            (bw, fw, aw), (bp, fp, ap) = whole[k], parts[k]
            for key in ("sun_rays", "ray_hits", "ray_stage_units", "intersections"):
                assert bw[key] == bp[key], (k, key)
            np.testing.assert_array_equal(fw, fp)
            np.testing.assert_array_equal(aw, ap)
    finally:
        for ctx in ctxs:
            product.st_free_context(ctx)
