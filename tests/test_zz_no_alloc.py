"""st_b200_probe_noalloc, the entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc: code inside a framework that owns
the device's memory, or a real-time loop that must not trigger the device-wide
synchronisation an allocation can cause.  It lists, in caller-owned device memory,
the sun rays of a range that hit the first stage, with the element they hit.

The check is against st_sim_run on the same scene and seed: ray numbers go to
first-stage hits in sun-ray order, so the k-th listed hit must be ray k's first
stage-1 element, and the last requested ray must come from sun ray SunRayCount - 1.
The entry point is called twice in a row, since calls share (and reuse) the static
scratch.  This file runs last so that a failure here stops no other test.
"""
import ctypes as C

import numpy as np
import pytest

from soltrace_b200 import scenes

pytestmark = pytest.mark.gpu

SIG = (C.c_int, [C.c_void_p, C.c_uint, C.c_ulonglong, C.c_uint, C.c_void_p, C.c_void_p,
                 C.POINTER(C.c_uint), C.c_void_p])


def _bind(api):
    fn = api.lib.st_b200_probe_noalloc
    fn.restype, fn.argtypes = SIG
    return fn


def _first_elements(rec, nrays):
    """|element| of each ray's first stage-1 record, in ray-number order."""
    s1 = rec["stage"] == 1
    rn, el = rec["raynum"][s1], np.abs(rec["element"][s1])
    first = np.zeros(nrays + 1, dtype=np.int64)
    seen = np.zeros(nrays + 1, dtype=bool)
    for r, e in zip(rn, el):  # readback order keeps each ray's hits in order
        if not seen[r]:
            seen[r] = True
            first[r] = e
    assert seen[1:].all()
    return first[1:]


@pytest.mark.parametrize("name", ["field", "dish"])
def test_probe_noalloc_matches_sim_run(product, name):
    import torch

    hits = 20000
    sc = scenes.field_scene(300, hits, dynamic_group=False) if name == "field" else scenes.dish_scene(hits)
    seed = 29
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_set_precision(ctx, 0)
        assert product.run(ctx, seed) > 0, product.messages(ctx)
        first = _first_elements(product.records(ctx), hits)
        nsun = product.sun_stats(ctx)["nsunrays"]

        probe = _bind(product)
        sid = torch.zeros(nsun, dtype=torch.int64, device="cuda")
        elem = torch.zeros(nsun, dtype=torch.int32, device="cuda")
        for call in range(2):
            sid.fill_(-1)
            elem.fill_(-1)
            torch.cuda.synchronize()
            nh = C.c_uint(0)
            rc = probe(ctx, seed, 0, nsun, sid.data_ptr(), elem.data_ptr(), C.byref(nh), None)
            assert rc == 1, product.messages(ctx)
            assert nh.value == hits, (call, nh.value)
            got_el = elem[:hits].cpu().numpy().astype(np.int64) + 1
            got_sid = sid[:hits].cpu().numpy()
            np.testing.assert_array_equal(got_el, first)
            assert int(got_sid[-1]) + 1 == nsun
            assert np.all(np.diff(got_sid) > 0)
    finally:
        product.st_free_context(ctx)


def test_probe_noalloc_rejects_oversized_requests(product):
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, scenes.dish_scene(100))
        nh = C.c_uint(7)
        rc = _bind(product)(ctx, 1, 0, (1 << 22) + 1, 16, 16, C.byref(nh), None)
        assert rc == -1 and nh.value == 0
        assert "at most" in product.messages(ctx)[-1]
    finally:
        product.st_free_context(ctx)


def test_probe_noalloc_rejects_explicit_ray_contexts(product):
    """A context given explicit rays traces those rays, not sun rays: the probe refuses it
    (before any device work) instead of listing sun rays st_sim_run would not trace."""
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, scenes.dish_scene(100))
        pos = np.array([[0.0, 0.0, 4.0]])
        cos = np.array([[0.0, 0.0, -1.0]])
        product.explicit_rays(ctx, pos, cos)
        nh = C.c_uint(7)
        rc = _bind(product)(ctx, 1, 0, 1000, 16, 16, C.byref(nh), None)
        assert rc == -1 and nh.value == 0
        assert "explicit rays" in product.messages(ctx)[-1]
    finally:
        product.st_free_context(ctx)
