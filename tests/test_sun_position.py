"""st_sun_position (no GPU): the product's against the reference's, bit for bit.

The front ends turn a date and time into a sun vector through st_sun_position
(coretrace/stapi.cpp:500-527) before calling st_sun_xyz; the product restates it on the
host.  scenes.sun_position, which the batched study's sun positions come from, follows the
same formula.
"""
import ctypes as C
import math

import numpy as np
import pytest


def _vec(api, lat, day, hour):
    x, y, z = C.c_double(), C.c_double(), C.c_double()
    assert api.st_sun_position(None, lat, day, hour, C.byref(x), C.byref(y), C.byref(z)) == 1
    return x.value, y.value, z.value


@pytest.fixture(scope="module")
def cases():
    rng = np.random.default_rng(4)
    return [(float(la), float(d), float(h)) for la, d, h in zip(rng.uniform(-60, 60, 400), rng.uniform(1, 365, 400),
                                                              rng.uniform(6, 18, 400))]


def test_matches_reference_bit_for_bit(product, reference, cases):
    for lat, day, hour in cases:
        assert _vec(product, lat, day, hour) == _vec(reference, lat, day, hour), (lat, day, hour)


def test_python_restatement_gives_the_same_sun(product, cases):
    from soltrace_b200 import scenes
    for lat, day, hour in cases:
        el, az = scenes.sun_position(lat, day, hour)
        d2r = math.pi / 180.0
        want = (-math.sin(az * d2r) * math.cos(el * d2r), math.sin(el * d2r), math.cos(az * d2r) * math.cos(el * d2r))
        np.testing.assert_allclose(_vec(product, lat, day, hour), want, rtol=0, atol=1e-12)
