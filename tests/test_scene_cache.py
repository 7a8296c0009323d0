"""A context reuses its flattened scene between runs only while the scene is unchanged.

st_sim_run skips the geometry set-up (grids, BVHs, beam lists) when a signature of every
scene input matches the last run's.  Any setter call that changes the scene must be seen:
after a change, the run must equal a fresh context's run of the changed scene.
"""
import numpy as np
import pytest

from soltrace_b200 import scenes

pytestmark = pytest.mark.gpu


def _run(api, ctx, seed):
    assert api.run(ctx, seed) > 0, api.messages(ctx)
    return api.records(ctx)


def _same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in a)


@pytest.mark.parametrize("change", ["move_absorber", "optic", "sun", "stage_flag", "aperture"])
def test_changed_scene_is_rebuilt(product, change):
    sc = scenes.dish_scene(5000)
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        first = _run(product, ctx, 5)
        again = _run(product, ctx, 5)
        assert _same(first, again)  # unchanged: the cached scene gives the same run
        if change == "move_absorber":
            product.st_element_xyz(ctx, 1, 0, 0.0, 0.0, 4.9)
            sc.stages[1].elements[0].origin = (0.0, 0.0, 4.9)
        elif change == "optic":
            o = sc.optics[0]
            o.front.slope = o.back.slope = 4.0
            scenes.push_optic(product, ctx, 0, o)
        elif change == "sun":
            product.st_sun_xyz(ctx, 1.0, 0.0, 100.0)
            sc.sun.xyz = (1.0, 0.0, 100.0)
        elif change == "stage_flag":
            product.st_stage_flags(ctx, 1, 0, 0, 0)
            sc.stages[1].multihit = False
        else:
            product.st_element_aperture(ctx, 1, 0, b"r")
            product.st_element_aperture_params(ctx, 1, 0, scenes.dptr(np.array([0.05, 0.05, 0, 0, 0, 0, 0, 0.0])))
            sc.stages[1].elements[0].aperture = "r"
            sc.stages[1].elements[0].aperture_params = (0.05, 0.05)
        changed = _run(product, ctx, 5)
    finally:
        product.st_free_context(ctx)
    fresh_ctx = product.st_create_context()
    try:
        scenes.push(product, fresh_ctx, sc)
        fresh = _run(product, fresh_ctx, 5)
    finally:
        product.st_free_context(fresh_ctx)
    assert _same(changed, fresh)
    if change != "stage_flag":  # the dish's absorber is met once per ray either way
        assert not _same(changed, first)
