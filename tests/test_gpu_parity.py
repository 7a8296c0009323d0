"""Parity of the CUDA trace (through the C ABI) with the CPU oracle and the reference.

* FP64, per ray: with the per-ray Philox streams the oracle and the device trace
  draw the same numbers, so every record must agree: element, stage and ray
  number exactly, positions within 1e-9 m (plus 2e-12 of the coordinate, the
  conditioning of the closed-form roots over km-scale paths), directions within
  1e-9.
* Mixed FP32/FP64, deterministic mode (explicit rays, errors off): same records,
  positions within 1e-5 m.
* Mixed vs FP64 GPU, statistical mode: flux-map L2 error <= 0.5 %.
* Device flux bins equal the oracle's bins from its records.
* Against the reference (a different random stream): intercept factors and flux
  totals within 3 sigma of the Monte-Carlo error.
"""
import numpy as np
import pytest

from helpers import assert_same_records, run_scene
from soltrace_b200 import scenes

pytestmark = pytest.mark.gpu

PHILOX = lambda a, c: a.st_oracle_set_rng(c, 1)  # noqa: E731


def _fp64(a, c):
    a.st_b200_set_precision(c, 0)


def _mixed(a, c):
    a.st_b200_set_precision(c, 1)


def _bench_scenes():
    return {
        "bench_dish": scenes.dish_scene(20000),
        "bench_trough": scenes.trough_scene(20000),
        "bench_field300": scenes.field_scene(300, 20000, dynamic_group=False),
        # the batched study's geometry: hyperboloid secondary, torus lip, ground receiver
        "bench_beam_down300": scenes.beam_down_scene(300, raycount=3000),
    }


ZOO_NAMES = ["sphere_circle", "sphere_line", "hyperboloid", "ellipsoid", "parabola_hex", "parabola_tri",
             "parabola_rect", "parabola_annulus", "parabola_irrtri", "parabola_quad", "trough_line", "cone",
             "general", "flat_circle", "torus", "torus_sector", "cylinder", "zernike", "poly", "spline", "vshot",
             "sun_gauss", "sun_table", "sun_point", "sun_oblique", "optics_pillbox", "optics_diffuse", "refl_table",
             "refraction", "virtual_stage", "tracethrough", "no_multihit", "multi_element", "fe_surface"]


@pytest.mark.parametrize("name", ZOO_NAMES + list(_bench_scenes()))
def test_fp64_matches_oracle_ray_by_ray(product, oracle, zoo_scenes, name):
    sc = zoo_scenes[name] if name in zoo_scenes else _bench_scenes()[name]
    a = run_scene(product, sc, 11, _fp64)
    b = run_scene(oracle, sc, 11, PHILOX)
    assert a[0] == b[0], (a[3], b[3])
    assert a[2] == b[2]  # sun box and SunRayCount
    # the finite-element surface interpolates with pow(), whose last bit differs between the
    # device and the host library; the Newton iteration on it then stops a step earlier or
    # later within its 1e-6 relative tolerance
    tol = 1e-7 if name == "fe_surface" else 1e-9
    if name == "bench_beam_down300":
        # The torus lip's quartic has coefficients built from pow(x, 4) terms, whose last bit
        # can differ between the device's pow and the host library's; the resolvent cubic's
        # bisection stops at a bracket width of 1e-6, so a flipped sign test moves the root
        # by up to about that much (4.1e-6 m measured on 76 of the 128 lip records, rays
        # starting tens of metres from the 0.5 m tube).  Every record's element, stage and
        # ray number is still identical, and every record off the lip is held to 1e-9 m.
        lip = (a[1]["stage"] == 2) & (np.abs(a[1]["element"]) == 2)
        assert lip.any()
        sub = lambda r, m: {k: v[m] for k, v in r.items()}  # noqa: E731
        assert_same_records(a[1], b[1], pos_tol=1e-5, dir_tol=1e-9)
        assert_same_records(sub(a[1], ~lip), sub(b[1], ~lip), pos_tol=tol, rel_tol=2e-12, dir_tol=tol)
        return
    assert_same_records(a[1], b[1], pos_tol=tol, rel_tol=2e-12, dir_tol=tol)


def _explicit_setup(pos, cos):
    def f(api, ctx):
        api.st_sim_errors(ctx, 0, 0)
        if hasattr(api, "st_b200_explicit_rays"):
            api.explicit_rays(ctx, pos, cos)
        else:
            from soltrace_b200.capi import dptr
            api.st_oracle_explicit_rays(ctx, len(pos), dptr(pos), dptr(cos))
    return f


@pytest.mark.parametrize("name", ["sphere_circle", "hyperboloid", "parabola_hex", "trough_line", "cylinder",
                                  "flat_circle", "refraction", "multi_element", "zernike", "spline", "torus"])
@pytest.mark.parametrize("prec", [0, 1])
def test_explicit_rays_deterministic(product, oracle, zoo_scenes, name, prec):
    """Deterministic mode: caller-supplied rays, errors off, reflectivity kept (the
    absorption draw uses the ray's own stream)."""
    sc = zoo_scenes[name]
    rng = np.random.default_rng(17)
    n = 4000
    pos = np.column_stack([rng.uniform(-2.5, 2.5, n), rng.uniform(-2.5, 2.5, n), np.full(n, 4.0)])
    d = np.column_stack([rng.normal(0, 0.05, n), rng.normal(0, 0.05, n), -np.ones(n)])
    cos = d / np.linalg.norm(d, axis=1)[:, None]

    def prod_setup(api, ctx):
        _explicit_setup(pos, cos)(api, ctx)
        api.st_b200_set_precision(ctx, prec)

    a = run_scene(product, sc, 5, prod_setup)
    b = run_scene(oracle, sc, 5, lambda x, c: (PHILOX(x, c), _explicit_setup(pos, cos)(x, c)))
    assert a[0] == b[0] > 0
    if prec == 0:
        assert_same_records(a[1], b[1], pos_tol=1e-9, rel_tol=2e-12, dir_tol=1e-9)
    else:
        assert_same_records(a[1], b[1], pos_tol=1e-5, dir_tol=1e-5)


def _flux_setup(prec, maps):
    def f(api, ctx):
        api.st_b200_set_precision(ctx, prec)
        for m in maps:
            api.st_b200_add_flux_map(ctx, *m)
    return f


DISH_MAP = (2, 1, 0, 50, 50, -0.25, 0.25, -0.25, 0.25, 1)


def _product_flux(product, sc, seed, prec, maps, records=True):
    ctx = product.st_create_context()
    scenes.push(product, ctx, sc)
    _flux_setup(prec, maps)(product, ctx)
    product.st_b200_set_records(ctx, 1 if records else 0)
    n = product.run(ctx, seed)
    assert n >= 0, product.messages(ctx)
    fl = [product.flux(ctx, i, m[3], m[4]) for i, m in enumerate(maps)]
    st = product.stats(ctx)
    product.st_free_context(ctx)
    return fl, st


def test_device_flux_bins_equal_oracle_bins(product, oracle):
    import ctypes as C
    sc = scenes.dish_scene(50000)
    fl, _ = _product_flux(product, sc, 3, 0, [DISH_MAP])
    ctx = oracle.st_create_context()
    scenes.push(oracle, ctx, sc)
    oracle.st_oracle_set_rng(ctx, 1)
    assert oracle.run(ctx, 3) > 0
    bins = np.zeros(50 * 50, dtype=np.uint64)
    oracle.st_oracle_flux(ctx, *DISH_MAP, bins.ctypes.data_as(C.POINTER(C.c_ulonglong)))
    oracle.st_free_context(ctx)
    np.testing.assert_array_equal(fl[0], bins.reshape(50, 50))


def test_records_off_keeps_flux_and_counts(product):
    sc = scenes.dish_scene(50000)
    on, st_on = _product_flux(product, sc, 4, 0, [DISH_MAP], records=True)
    off, st_off = _product_flux(product, sc, 4, 0, [DISH_MAP], records=False)
    np.testing.assert_array_equal(on[0], off[0])
    assert st_on["sun_rays"] == st_off["sun_rays"] and st_off["records"] == 0


def test_mixed_flux_within_half_percent_of_fp64(product):
    """The benchmark metric's accuracy bar: flux-map L2 error of the mixed trace
    against the FP64 device trace <= 0.5 %."""
    sc = scenes.dish_scene(400000)
    f64, _ = _product_flux(product, sc, 9, 0, [DISH_MAP], records=False)
    fmx, _ = _product_flux(product, sc, 9, 1, [DISH_MAP], records=False)
    a, b = f64[0].astype(float), fmx[0].astype(float)
    l2 = np.linalg.norm(a - b) / np.linalg.norm(a)
    assert l2 <= 0.005, l2


def test_field_mixed_flux_within_half_percent(product):
    sc = scenes.field_scene(300, 200000, dynamic_group=False)
    m = (2, 1, 1, 72, 40, 0.0, 4.0, -5.0, 5.0, 1)
    f64, _ = _product_flux(product, sc, 9, 0, [m], records=False)
    fmx, _ = _product_flux(product, sc, 9, 1, [m], records=False)
    a, b = f64[0].astype(float), fmx[0].astype(float)
    assert np.linalg.norm(a - b) / np.linalg.norm(a) <= 0.005


def _intercept(rec, target_stage, first_stage=1):
    hits1 = len(np.unique(rec["raynum"][rec["stage"] == first_stage]))
    absorbed = int(np.sum((rec["stage"] == target_stage) & (rec["element"] < 0)))
    return absorbed / hits1, hits1


@pytest.mark.parametrize("sc_name", ["dish", "trough"])
def test_statistics_match_reference(product, reference, sc_name):
    """Different random streams: per-stage absorbed fractions agree within 3 sigma."""
    sc = scenes.dish_scene(200000) if sc_name == "dish" else scenes.trough_scene(200000)
    a = run_scene(product, sc, 21, _fp64)[1]
    b = run_scene(reference, sc, 21)[1]
    for s in sorted(set(b["stage"].tolist())):
        pa = np.mean((a["stage"] == s) & (a["element"] < 0)) * len(a["x"]) / 200000
        pb = np.mean((b["stage"] == s) & (b["element"] < 0)) * len(b["x"]) / 200000
        sig = np.sqrt(max(pb * (1 - pb), 1e-12) / 200000) * np.sqrt(2)
        assert abs(pa - pb) <= 3 * sig + 1e-12, (s, pa, pb, sig)


def test_per_heliostat_counts(product):
    sc = scenes.field_scene(120, 50000, dynamic_group=False)
    ctx = product.st_create_context()
    scenes.push(product, ctx, sc)
    assert product.run(ctx, 2) > 0
    rec = product.records(ctx)
    first, absorbed, delivered = product.element_counts(ctx, 1, 120)
    st = product.stats(ctx)
    product.st_free_context(ctx)
    # first hits per heliostat = distinct rays whose first stage-1 record is that heliostat
    s1 = rec["stage"] == 1
    order = np.lexsort((np.arange(len(rec["x"]))[s1], rec["raynum"][s1]))
    rn, el = rec["raynum"][s1][order], np.abs(rec["element"][s1][order])
    firsts = el[np.r_[True, rn[1:] != rn[:-1]]]
    np.testing.assert_array_equal(first, np.bincount(firsts - 1, minlength=120))
    assert int(delivered.sum()) == int(np.sum((rec["stage"] == 2) & (rec["element"] < 0)))
    assert st["ray_hits"] == 50000 and st["sun_rays"] >= 50000


@pytest.mark.parametrize("prec", [0, 1])
def test_sun_ray_cap_fails_like_the_oracle(product, oracle, prec):
    """A run that needs more sun rays than st_sim_params' maximum returns -1 with the
    reference's message (raytrace.cpp:600-602; the oracle's message is pinned to the
    reference's in test_oracle.py), and the context runs again once the cap is raised."""
    tight = scenes.dish_scene(1000)
    tight.raymax = 500
    want = run_scene(oracle, tight, 1)
    assert want[0] == -1
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, tight)
        product.st_b200_set_precision(ctx, prec)
        assert product.run(ctx, 1) == -1
        assert want[3][-1] in product.messages(ctx), (product.messages(ctx), want[3])
        product.st_sim_params(ctx, 1000, 1_000_000, 0)
        assert product.run(ctx, 1) > 0, product.messages(ctx)
        assert product.stats(ctx)["ray_hits"] == 1000
    finally:
        product.st_free_context(ctx)
