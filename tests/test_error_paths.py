"""Failure paths the front ends show to users (no GPU): return codes and messages of the
product equal the reference's.  Every case fails in scene set-up, before any device work,
so the product answers here without a GPU exactly as it does on a B200."""
import copy

import pytest

from helpers import run_scene
from soltrace_b200 import scenes


def _broken():
    base = scenes.dish_scene(100)
    out = {}
    s = copy.deepcopy(base)
    s.stages[0].elements[0].optic = "missing"
    out["unknown optic"] = s
    s = copy.deepcopy(base)
    s.stages = []
    out["no stages"] = s
    s = copy.deepcopy(base)
    s.stages[0].elements = []
    out["first stage empty"] = s
    s = copy.deepcopy(base)
    s.raycount = 0
    out["no rays"] = s
    return out


@pytest.mark.parametrize("case", sorted(_broken()))
def test_run_fails_with_the_reference_message(product, reference, case):
    sc = _broken()[case]
    a = run_scene(product, sc, 1)
    b = run_scene(reference, sc, 1)
    assert a[0] == b[0] == -1
    assert a[3] == b[3], (a[3], b[3])


def test_missing_surface_file_fails_with_the_reference_message(product, reference):
    sc = scenes.dish_scene(100)
    res = []
    for api in (product, reference):
        ctx = api.st_create_context()
        try:
            scenes.push(api, ctx, sc)
            rc = api.st_element_surface_file(ctx, 0, 0, b"/nonexistent/surface.mon")
            res.append((rc, api.messages(ctx)))
        finally:
            api.st_free_context(ctx)
    assert res[0][0] == res[1][0] == -1
    assert res[0][1] == res[1][1], res
