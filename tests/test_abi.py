"""The C-ABI boundary of coretrace_api.so, checked without a GPU.

Every function declared in include/*.h is exported; setters follow the
reference's return conventions; without a CUDA device st_sim_run fails loudly
(-1 and a message) instead of falling back to anything.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from soltrace_b200 import scenes
from soltrace_b200.capi import STAPI_FUNCTIONS, dptr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"\b(st_[a-z0-9_]+)\s*\(", txt))


def _exports():
    lib = os.path.join(ROOT, "soltrace_b200", "coretrace_api.so")
    if not os.path.exists(lib):
        pytest.skip("coretrace_api.so not built")
    out = os.popen(f"nm -D --defined-only {lib}").read()
    return set(re.findall(r" T (st_[a-z0-9_]+)", out))


def test_every_declared_function_is_exported():
    exported = _exports()
    for h in ("stapi.h", "st_b200.h"):
        missing = _declared(h) - exported
        assert not missing, (h, missing)


def test_stapi_header_matches_reference_declarations():
    """Every function the reference's coretrace/stapi.h declares (tests/golden/
    reference_stapi.json, parsed from it by tests/golden/make_api_fixture.py) is declared in
    include/stapi.h with the same return and parameter types, and exported."""
    import json

    from helpers import c_declarations
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_stapi.json")))["functions"]
    assert len(ref) >= 50
    mine = c_declarations(open(os.path.join(ROOT, "include", "stapi.h")).read())
    exported = _exports()
    for name, d in ref.items():
        assert name in mine, name
        assert mine[name] == (d["returns"], d["params"]), (name, mine[name], d)
        assert name in exported, name
    # the ctypes table used by the tests binds the same set
    assert set(STAPI_FUNCTIONS) == set(ref)


def test_batch_arguments_checked_before_device_work(product):
    """st_b200_sim_run_batch rejects bad arguments and explicit-ray contexts with -1 and a
    message, before touching a device."""
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, scenes.dish_scene(100))
        assert product.run_batch(ctx, 1, np.zeros((0, 3)), []) == -1
        assert "at least one sun position" in product.messages(ctx)[-1]
        product.explicit_rays(ctx, np.array([[0.0, 0.0, 4.0]]), np.array([[0.0, 0.0, -1.0]]))
        assert product.run_batch(ctx, 1, np.array([[0.0, 0.0, 100.0]]), [10]) == -1
        assert "explicit rays" in product.messages(ctx)[-1]
        assert product.st_b200_batch_stats(ctx, 0, None) == -1
    finally:
        product.st_free_context(ctx)


def test_library_loads_and_setters(product):
    api = product
    ctx = api.st_create_context()
    assert ctx
    assert api.st_add_stage(ctx) == 0
    assert api.st_add_stages(ctx, 2) == 2
    assert api.st_num_stages(ctx) == 3
    assert api.st_add_elements(ctx, 0, 4) == 4
    assert api.st_add_element(ctx, 0) == 4
    assert api.st_num_elements(ctx, 0) == 5
    assert api.st_element_xyz(ctx, 0, 9, 0.0, 0.0, 0.0) == -1  # bad element index
    assert api.st_stage_xyz(ctx, 7, 0.0, 0.0, 0.0) == -1  # bad stage index
    assert api.st_delete_element(ctx, 0, 1) == 1
    assert api.st_num_elements(ctx, 0) == 4
    assert api.st_add_optic(ctx, b"a") == 0 and api.st_add_optic(ctx, b"b") == 1
    assert api.st_num_optics(ctx) == 2
    # cylinder surface needs an 'l' aperture with A = B = 0 (input.cpp:339-343)
    api.st_element_aperture(ctx, 0, 0, b"c")
    api.st_element_surface(ctx, 0, 0, b"t")
    p = np.zeros(8)
    p[0] = 0.5
    assert api.st_element_surface_params(ctx, 0, 0, dptr(p)) == -1
    assert "cylindrical" in api.messages(ctx)[-1]
    api.st_clear_messages(ctx)
    assert api.st_num_messages(ctx) == 0
    assert api.st_sun_userdata(ctx, 2, dptr(np.zeros(2)), dptr(np.zeros(2))) == -1
    assert api.st_free_context(ctx) == 1


def test_transform_utilities_match_oracle(product, oracle):
    rng = np.random.default_rng(0)
    for _ in range(20):
        o, a = rng.normal(size=3), rng.normal(size=3) * 10
        z = float(rng.uniform(-180, 180))
        e1, e2 = np.zeros(3), np.zeros(3)
        product.st_calc_euler_angles(dptr(o), dptr(a), z, dptr(e1))
        # oracle side: same Euler formula via st_element geometry is internal; compare with numpy
        d = (a - o) / np.linalg.norm(a - o)
        e2[:] = [np.arctan2(d[0], d[2]), np.arcsin(d[1]), z * 0.017453292519943295]
        np.testing.assert_allclose(e1, e2, rtol=0, atol=1e-15)
        R1, R1t = np.zeros((3, 3)), np.zeros((3, 3))
        product.st_calc_transform_matrices(dptr(e1), dptr(R1), dptr(R1t))
        np.testing.assert_array_equal(R1t, R1.T)
        np.testing.assert_allclose(R1 @ R1.T, np.eye(3), atol=1e-14)


def test_run_without_gpu_fails_loudly(product):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    ctx = product.st_create_context()
    scenes.push(product, ctx, scenes.dish_scene(100))
    assert product.run(ctx, 1) == -1
    assert any("CUDA" in m for m in product.messages(ctx))
    # the batched entry point too, before it stages anything
    assert product.run_batch(ctx, 1, np.array([[0.0, 0.0, 100.0], [0.0, 50.0, 100.0]]), [10, 10]) == -1
    assert "CUDA" in product.messages(ctx)[-1]
    product.st_free_context(ctx)


def test_geometry_errors_reported_before_any_device_work(product):
    sc = scenes.dish_scene(100)
    sc.stages[0].elements[0].optic = "missing"
    ctx = product.st_create_context()
    scenes.push(product, ctx, sc)
    assert product.run(ctx, 1) == -1
    assert "invalid optical property set name" in product.messages(ctx)[0]
    product.st_free_context(ctx)


def test_fused_forward_rejects_unsupported_shapes(product):
    """The fused forward's shape rules are checked on the host (no device needed)."""
    fn = product.lib.st_b200_mlp_packed_bytes
    fn.restype, fn.argtypes = C.c_longlong, [C.c_int, C.c_void_p]
    for dims in [(8, 128, 256), (32, 256, 256), (8, 256, 300), (8, 256), (8,) + (256,) * 9]:
        arr = (C.c_int * len(dims))(*dims)
        assert fn(len(dims) - 1, arr) == -1, dims
    arr = (C.c_int * 4)(8, 256, 256, 1024)
    assert fn(3, arr) == 2 * (4096 + 16384 * (4 + 16))
