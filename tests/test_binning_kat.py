"""The trough example's receiver binning (flux-map kind 4) against the reference's own code.

* The known-answer test of the example's test suite
  (app/deploy/api/examples/parabolic-trough-tracking-timeseries/tests/test_flux_map.py:51-68):
  three hand-placed points on the absorber tube -- its leftmost, lowest and rightmost points --
  binned on a 5 x 4 and a 5 x 3 mesh give flux 0.90945591 (5 x 4) and 0.68209193 (5 x 3) in
  three bins (power per ray 10, flux = count x ppr / node area x 1e-3).
* Fixtures made by the example's own functions (tests/golden/make_binning_fixtures.py): random
  points on tubes of several radii, lengths and mesh sizes (odd and even, one-cell meshes,
  points beyond the tube ends, the even-mesh tie at y = 0) binned by compute_fluxmap; the
  oracle's kind-4 rule gives the same count grids.
The device's kind-4 maps are compared with the oracle's on a traced trough
(tests/test_flux_stats.py).
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
R_KAT = 1 / 28.5714
KAT = {  # (nx, ny) -> the published flux grid [ix][iy]
    (5, 4): np.array([[0., 0., 0., 0.], [0., 0.90945591, 0., 0.], [0., 0., 0., 0.], [0., 0.90945591, 0., 0.],
                      [0., 0.90945591, 0., 0.]]),
    (5, 3): np.array([[0., 0., 0.], [0., 0.68209193, 0.], [0., 0., 0.], [0., 0.68209193, 0.], [0., 0.68209193, 0.]]),
}


def _bin(oracle, r, l, nx, ny, pts):
    fn = oracle.lib.st_oracle_bin_point
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_double] * 7 + [C.POINTER(C.c_int), C.POINTER(C.c_int)]
    counts = np.zeros((nx, ny), dtype=np.int64)
    ix, iy = C.c_int(), C.c_int()
    for x, y, z in pts:
        assert fn(4, nx, ny, 0.0, r, -l / 2, l / 2, x, y, z, C.byref(ix), C.byref(iy)) == 1
        counts[ix.value, iy.value] += 1
    return counts


@pytest.mark.parametrize("mesh", sorted(KAT))
def test_known_answer_of_the_trough_example(oracle, mesh):
    nx, ny = mesh
    r, l = R_KAT, 1.0
    # leftmost, lowest and rightmost points of the tube, element-local (axis at z = r)
    pts = [(-r, 0.0, r), (0.0, 0.0, 0.0), (r, 0.0, r)]
    counts = _bin(oracle, r, l, nx, ny, pts)
    dx, dy = math.pi * (2 * r) / nx, l / ny
    flux = counts * (10.0 / (dx * dy) * 1e-3)
    assert np.allclose(flux, KAT[mesh])


def test_binning_equals_the_example_functions(oracle):
    with open(os.path.join(HERE, "golden", "reference_binning.json")) as f:
        cases = json.load(f)["cases"]
    assert len(cases) == 8
    for c in cases:
        got = _bin(oracle, c["r"], c["l"], c["nx"], c["ny"], c["points"])
        np.testing.assert_array_equal(got, np.array(c["counts"]), err_msg=f"{c['nx']}x{c['ny']} r={c['r']}")
