"""The stapi.h setters (no GPU): one script of valid and out-of-range calls applied to the
product and to the reference gives the same return codes, the same counts and the same
messages after every call."""
import numpy as np

from soltrace_b200.capi import dptr


def _script(api, ctx):
    """(call, return code) pairs, then counts, in order."""
    p8 = np.array([1.0, 2.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0])
    calls = [
        ("add_optic", lambda: api.st_add_optic(ctx, b"mirror")),
        ("add_stages", lambda: api.st_add_stages(ctx, 2)),
        ("add_elements", lambda: api.st_add_elements(ctx, 0, 3)),
        ("add_element", lambda: api.st_add_element(ctx, 1)),
        ("stage_xyz ok", lambda: api.st_stage_xyz(ctx, 1, 0.0, 0.0, 5.0)),
        ("stage_xyz bad", lambda: api.st_stage_xyz(ctx, 7, 0.0, 0.0, 5.0)),
        ("stage_aim bad", lambda: api.st_stage_aim(ctx, 2, 0.0, 0.0, 1.0)),
        ("stage_zrot ok", lambda: api.st_stage_zrot(ctx, 0, 12.0)),
        ("stage_flags bad", lambda: api.st_stage_flags(ctx, 3, 0, 1, 0)),
        ("element_xyz ok", lambda: api.st_element_xyz(ctx, 0, 2, 1.0, 2.0, 3.0)),
        ("element_xyz bad elem", lambda: api.st_element_xyz(ctx, 0, 3, 1.0, 2.0, 3.0)),
        ("element_xyz bad stage", lambda: api.st_element_xyz(ctx, 5, 0, 1.0, 2.0, 3.0)),
        ("element_aim bad", lambda: api.st_element_aim(ctx, 1, 1, 0.0, 0.0, 1.0)),
        ("element_zrot ok", lambda: api.st_element_zrot(ctx, 1, 0, 30.0)),
        ("element_enabled bad", lambda: api.st_element_enabled(ctx, 0, 9, 0)),
        ("aperture ok", lambda: api.st_element_aperture(ctx, 0, 0, b"r")),
        ("aperture bad", lambda: api.st_element_aperture(ctx, 0, 4, b"r")),
        ("aperture params ok", lambda: api.st_element_aperture_params(ctx, 0, 0, dptr(p8))),
        ("surface bad", lambda: api.st_element_surface(ctx, 2, 0, b"s")),
        ("surface params bad", lambda: api.st_element_surface_params(ctx, 0, 8, dptr(p8))),
        ("interaction ok", lambda: api.st_element_interaction(ctx, 0, 1, 2)),
        ("interaction bad", lambda: api.st_element_interaction(ctx, 1, 5, 2)),
        ("optic name ok", lambda: api.st_element_optic(ctx, 0, 0, b"mirror")),
        ("optic name bad index", lambda: api.st_element_optic(ctx, 0, 7, b"mirror")),
        ("delete element bad", lambda: api.st_delete_element(ctx, 0, 5)),
        ("delete element ok", lambda: api.st_delete_element(ctx, 0, 1)),
        ("clear elements bad", lambda: api.st_clear_elements(ctx, 4)),
        ("delete stage bad", lambda: api.st_delete_stage(ctx, 9)),
        ("delete optic bad", lambda: api.st_delete_optic(ctx, 3)),
        ("delete stage ok", lambda: api.st_delete_stage(ctx, 1)),
        ("sim params", lambda: api.st_sim_params(ctx, 100, 1000, 0)),
        ("sim errors", lambda: api.st_sim_errors(ctx, 1, 0)),
        ("sun", lambda: api.st_sun(ctx, 0, b"g", 2.5)),
        ("sun xyz", lambda: api.st_sun_xyz(ctx, 0.0, 0.0, 100.0)),
    ]
    out = []
    for name, f in calls:
        rc = f()
        counts = (api.st_num_stages(ctx), api.st_num_optics(ctx),
                  [api.st_num_elements(ctx, s) for s in range(max(api.st_num_stages(ctx), 0))])
        out.append((name, rc, counts, api.messages(ctx)))
    return out


def test_setters_match_reference(product, reference):
    res = []
    for api in (product, reference):
        ctx = api.st_create_context()
        try:
            res.append(_script(api, ctx))
        finally:
            api.st_free_context(ctx)
    for a, b in zip(*res):
        assert a == b, (a, b)
