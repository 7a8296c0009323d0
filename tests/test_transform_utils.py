"""stapi.h's transform utilities (no GPU): the product's against the reference's, bit for bit.

st_calc_euler_angles, st_calc_transform_matrices, st_transform_to_local,
st_transform_to_reference, st_matrix_vector_mult and st_matrix_transpose are the geometry
helpers front ends call directly (coretrace/stapi.cpp, mathproc.cpp:58-217); the device's
frames are built from the same arithmetic.
"""
import numpy as np

from soltrace_b200.capi import dptr


def _pair(product, reference, fn, *args, outs):
    res = []
    for api in (product, reference):
        bufs = [np.zeros(n) for n in outs]
        getattr(api, fn)(*[dptr(a) if isinstance(a, np.ndarray) else a for a in args], *[dptr(b) for b in bufs])
        res.append(bufs)
    for x, y in zip(*res):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), (fn, x, y)
    return res[0]


def test_transform_utilities_match_reference(product, reference):
    rng = np.random.default_rng(8)
    for _ in range(200):
        o = rng.normal(size=3) * 100.0
        a = o + rng.normal(size=3) * 50.0
        z = float(rng.uniform(-180, 180))
        (eu,) = _pair(product, reference, "st_calc_euler_angles", o.copy(), a.copy(), z, outs=[3])
        r2l, l2r = _pair(product, reference, "st_calc_transform_matrices", eu.copy(), outs=[9, 9])
        p, c = rng.normal(size=3) * 500.0, rng.normal(size=3)
        c /= np.linalg.norm(c)
        _pair(product, reference, "st_transform_to_local", p.copy(), c.copy(), o.copy(), r2l.copy(), outs=[3, 3])
        _pair(product, reference, "st_transform_to_reference", p.copy(), c.copy(), o.copy(), l2r.copy(), outs=[3, 3])
        _pair(product, reference, "st_matrix_vector_mult", r2l.copy(), p.copy(), outs=[3])
        _pair(product, reference, "st_matrix_transpose", r2l.copy(), outs=[9])
