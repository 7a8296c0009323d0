"""Flux maps with the SolTrace GUI's binning rules and the GUI's element flux statistics.

Kinds 2 and 3 of st_b200_add_flux_map bin as the GUI's ElementStatistics does
(app/src/project.cpp:1300-1419): bins (lower, upper] found by its increment loop, and for a
full cylinder the unwrapped arc length.  The device maps must equal the oracle's bins
ray for ray (FP64, per-ray streams), and st_b200_flux_stats must return the GUI's
statistics (project.cpp:1240-1288) of those counts.
"""
import ctypes as C
import math

import numpy as np
import pytest

from soltrace_b200 import scenes

pytestmark = pytest.mark.gpu

DISH_GUI = (2, 1, 2, 40, 30, -0.25, 0.25, -0.25, 0.25, 1)          # flat receiver disc
DISH_PYS = (2, 1, 0, 40, 30, -0.25, 0.25, -0.25, 0.25, 1)
FIELD_GUI = (2, 1, 3, 64, 20, 0.0, 4.0, -5.0, 5.0, 1)              # cylinder, radius 4
FIELD_PYS = (2, 1, 1, 64, 20, 0.0, 4.0, -5.0, 5.0, 1)


def _product(product, sc, seed, maps):
    ctx = product.st_create_context()
    scenes.push(product, ctx, sc)
    product.st_b200_set_precision(ctx, 0)
    for m in maps:
        assert product.st_b200_add_flux_map(ctx, *m) >= 0
    assert product.run(ctx, seed) > 0, product.messages(ctx)
    return ctx


def _oracle_bins(oracle, sc, seed, m):
    ctx = oracle.st_create_context()
    scenes.push(oracle, ctx, sc)
    oracle.st_oracle_set_rng(ctx, 1)
    assert oracle.run(ctx, seed) > 0
    bins = np.zeros(m[3] * m[4], dtype=np.uint64)
    oracle.st_oracle_flux(ctx, *m, bins.ctypes.data_as(C.POINTER(C.c_ulonglong)))
    oracle.st_free_context(ctx)
    return bins.reshape(m[4], m[3])


def _gui_stats(counts, ppr, bx, by, intersections):
    """project.cpp:1240-1288 on a [iy][ix] count grid (x-major scan for peak and minimum)."""
    nx, ny = counts.shape[1], counts.shape[0]
    zs = ppr / (bx * by)
    peak, mn, npk, s, s2 = 0.0, 1e99, None, 0.0, 0.0
    for ix in range(nx):
        for iy in range(ny):
            z = float(counts[iy, ix]) * zs
            s += z
            s2 += z * z
            if z > peak:
                peak, npk = z, int(counts[iy, ix])
            if z < mn:
                mn = z
    n = nx * ny
    ave = s / n
    sig = math.sqrt((n * s2 - s * s) / (n * n))
    return {"peak_flux": peak, "min_flux": mn, "ave_flux": ave, "sigma_flux": sig, "uniformity": sig / ave,
            "peak_flux_uncertainty": 100 / math.sqrt(npk), "ave_flux_uncertainty": 100 / math.sqrt(intersections)}


@pytest.mark.parametrize("case", ["dish", "field"])
def test_gui_bins_equal_oracle_and_stats_match(product, oracle, case):
    if case == "dish":
        sc, gui, pys, dni = scenes.dish_scene(60000), DISH_GUI, DISH_PYS, 1000.0
        bx, by = 0.5 / gui[3], 0.5 / gui[4]
    else:
        sc, gui, pys, dni = scenes.field_scene(300, 100000, dynamic_group=False), FIELD_GUI, FIELD_PYS, 950.0
        bx, by = 2 * math.pi * 4.0 / gui[3], 10.0 / gui[4]
    seed = 11
    ctx = _product(product, sc, seed, [gui, pys])
    try:
        g = product.flux(ctx, 0, gui[3], gui[4])
        p = product.flux(ctx, 1, pys[3], pys[4])
        np.testing.assert_array_equal(g, _oracle_bins(oracle, sc, seed, gui))
        # every absorbed hit inside the y range lands in a bin under both rules, except a
        # point whose |x| rounds above the cylinder radius: the GUI's asin(x/R) is NaN there
        # and the GUI leaves it unbinned
        assert p.sum() > 0 and abs(int(g.sum()) - int(p.sum())) <= 2
        st = product.flux_stats(ctx, 0, dni)
        sun = product.sun_stats(ctx)
        ppr = dni * (sun["xmax"] - sun["xmin"]) * (sun["ymax"] - sun["ymin"]) / sun["nsunrays"]
        want = _gui_stats(g, ppr, bx, by, len(product.records(ctx)["raynum"]))
        assert st["power_per_ray"] == pytest.approx(ppr, rel=1e-12)
        assert st["bin_area"] == pytest.approx(bx * by, rel=1e-12)
        for k, v in want.items():
            assert st[k] == pytest.approx(v, rel=1e-9), k
        assert st["rays_binned"] == int(g.sum())
    finally:
        product.st_free_context(ctx)


@pytest.mark.parametrize("mesh", [(72, 120), (5, 4), (1, 3)])
def test_trough_mesh_bins_equal_oracle(product, oracle, mesh):
    """Kind 4, the trough example's nearest-node rule on the absorber tube (radius 35 mm,
    12 m), on the device against the oracle's restatement of the example's functions (pinned
    to them in tests/test_binning_kat.py): the same rays land in the same nodes; every
    absorbed hit is binned."""
    nx, ny = mesh
    m = (3, 2, 4, nx, ny, 0.0, 0.035, -6.0, 6.0, 1)
    sc = scenes.trough_scene(40000)
    ctx = _product(product, sc, 9, [m])
    try:
        got = product.flux(ctx, 0, nx, ny)
        rec = product.records(ctx)
        absorbed = int(np.sum((np.asarray(rec["stage"]) == 3) & (np.asarray(rec["element"]) == -2)))
    finally:
        product.st_free_context(ctx)
    np.testing.assert_array_equal(got, _oracle_bins(oracle, sc, 9, m))
    assert got.sum() == absorbed > 0


def test_flux_stats_without_records_counts_intersections(product):
    """With records off the run still counts its intersections for the mean-flux uncertainty."""
    sc = scenes.dish_scene(30000)
    out = []
    for rec in (1, 0):
        ctx = product.st_create_context()
        scenes.push(product, ctx, sc)
        product.st_b200_set_records(ctx, rec)
        product.st_b200_add_flux_map(ctx, *DISH_GUI)
        assert product.run(ctx, 5) >= 0, product.messages(ctx)
        out.append((product.flux_stats(ctx, 0, 1000.0), product.stats(ctx)))
        product.st_free_context(ctx)
    (a, sa), (b, sb) = out
    assert sa["records"] > 0 and sb["records"] == 0
    assert sb["intersections"] == sa["intersections"] == sa["records"]
    assert a == b


def test_flux_stats_rejects_bad_requests(product):
    ctx = product.st_create_context()
    try:
        scenes.push(product, ctx, scenes.dish_scene(100))
        assert product.st_b200_add_flux_map(ctx, 2, 1, 5, 10, 10, 0.0, 1.0, 0.0, 1.0, 1) == -1  # kind
        assert product.st_b200_add_flux_map(ctx, 2, 1, 4, 10, 10, 0.0, 0.0, 0.0, 1.0, 1) == -1  # radius
        assert product.st_b200_add_flux_map(ctx, 2, 1, 2, 10, 10, 1.0, 0.0, 0.0, 1.0, 1) == -1  # x range
        m = product.st_b200_add_flux_map(ctx, *DISH_GUI)
        with pytest.raises(RuntimeError):
            product.flux_stats(ctx, m, 1000.0)  # no run yet
    finally:
        product.st_free_context(ctx)
