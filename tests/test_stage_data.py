"""Stage-data save and replay (st_b200_set_save_stage_data, st_b200_stage_data,
st_b200_sim_run_replay): the C form of the reference's st_sim_run_data
(coretrace/stapi.cpp:680-728).

Pin: stage data saved by the reference itself (its st_sim_run_data, called through the
C harness oracle/ref_stage_data.cpp built with the reference's objects) are replayed by the
reference and by the product; on the dish, whose second stage is a pure absorber (its
outcome needs no random draw), both replays give the same records.  The product's own
save / replay round trip reproduces its run, and the saved second-stage input follows the
reference's in-place layout.
"""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import assert_same_records
from soltrace_b200 import scenes
from soltrace_b200.capi import StApi, c_double_p

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SD = os.path.join(ROOT, "oracle", "_ref", "coretrace_ref_sd.so")
SD_EXTRA = {
    "ref_sd_run_save": (C.c_int, [C.c_void_p, C.c_uint]),
    "ref_sd_sizes": (C.c_int, [C.POINTER(C.c_ulong), C.POINTER(C.c_ulong)]),
    "ref_sd_get": (C.c_int, [c_double_p, c_double_p]),
    "ref_sd_run_replay": (C.c_int, [C.c_void_p, C.c_uint, C.c_ulong, c_double_p, C.c_ulong, c_double_p]),
}


@pytest.fixture(scope="module")
def ref_sd():
    if not os.path.exists(REF_SD):
        pytest.skip("reference stage-data harness not built (make -C oracle ref)")
    return StApi(REF_SD, SD_EXTRA)


def _ref_save(ref, sc, seed):
    ctx = ref.st_create_context()
    scenes.push(ref, ctx, sc)
    assert ref.ref_sd_run_save(ctx, seed) > 0, ref.messages(ctx)
    rec = ref.records(ctx)
    ref.st_free_context(ctx)
    n0, n1 = C.c_ulong(), C.c_ulong()
    ref.ref_sd_sizes(C.byref(n0), C.byref(n1))
    s0, s1 = np.zeros((n0.value, 8)), np.zeros((n1.value, 7))
    ref.ref_sd_get(s0.ctypes.data_as(c_double_p), s1.ctypes.data_as(c_double_p))
    return s0, s1, rec


def _ref_replay(ref, sc, seed, s0, s1):
    ctx = ref.st_create_context()
    scenes.push(ref, ctx, sc)
    s0c, s1c = np.ascontiguousarray(s0), np.ascontiguousarray(s1)
    n = ref.ref_sd_run_replay(ctx, seed, len(s0c), s0c.ctypes.data_as(c_double_p), len(s1c),
                              s1c.ctypes.data_as(c_double_p))
    assert n > 0, ref.messages(ctx)
    rec, sun = ref.records(ctx), ref.sun_stats(ctx)
    ref.st_free_context(ctx)
    return rec, sun


def _product_run(product, sc, seed, save=False, replay=None):
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, sc)
        product.st_b200_set_precision(ctx, 0)
        product.st_b200_set_save_stage_data(ctx, int(save))
        n = product.run_replay(ctx, seed, *replay) if replay else product.run(ctx, seed)
        assert n > 0, product.messages(ctx)
        return product.records(ctx), product.sun_stats(ctx), (product.stage_data(ctx) if save else None)
    finally:
        product.st_free_context(ctx)


def test_replay_of_reference_saved_data_matches_reference_replay(product, ref_sd):
    sc = scenes.dish_scene(20000)
    s0, s1, _ = _ref_save(ref_sd, sc, 7)
    assert len(s0) > 0 and len(s1) > 0
    want, want_sun = _ref_replay(ref_sd, sc, 8, s0, s1)
    got, got_sun, _ = _product_run(product, sc, 8, replay=(s0, s1))
    assert got_sun["nsunrays"] == want_sun["nsunrays"] == int(s0[-1, 7])
    assert_same_records(got, want, 1e-9, rel_tol=2e-12, dir_tol=1e-12)


def test_product_save_replay_round_trip(product):
    sc = scenes.dish_scene(20000)
    rec, sun, (s0, s1) = _product_run(product, sc, 5, save=True)
    st1 = rec["stage"] == 1
    np.testing.assert_array_equal(s0[:, 7], rec["raynum"][st1])
    np.testing.assert_array_equal(s0[:, 6], rec["element"][st1])
    np.testing.assert_array_equal(s0[:, 0], rec["x"][st1])
    # the second stage absorbs everything: the saved input is the rays entering it
    assert len(s1) == len(np.unique(rec["raynum"][rec["stage"] == 2]))
    rec2, sun2, _ = _product_run(product, sc, 99, replay=(s0, s1))
    assert sun2["nsunrays"] == int(s0[-1, 7])
    for k in rec:
        np.testing.assert_array_equal(rec2[k], rec[k], err_msg=k)


def test_saved_second_stage_input_keeps_the_reference_layout(product):
    """Trough: rays leave the second stage (outer glass) for the third, so the saved input
    starts with the rays that left it and continues with the rays that entered it."""
    sc = scenes.trough_scene(20000)
    rec, _, (s0, s1) = _product_run(product, sc, 3, save=True)
    entered = np.unique(rec["raynum"][rec["stage"] == 2])
    left = np.unique(rec["raynum"][rec["stage"] == 3])  # every ray entering stage 3 leaves a record
    w = len(left)
    assert 0 < w < len(entered)
    want = np.concatenate([left, entered[w:]]).astype(float)
    np.testing.assert_array_equal(s1[:, 6], want)


def test_replay_without_data_traces_from_the_sun(product):
    sc = scenes.dish_scene(3000)
    a, _, _ = _product_run(product, sc, 4)
    b, _, _ = _product_run(product, sc, 4, replay=(np.zeros((0, 8)), np.zeros((0, 7))))
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
