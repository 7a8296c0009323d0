"""Host logic of the flux surrogate's inputs (no GPU): the 16 situation features.

The bench evaluates them with numpy, the aim optimiser with torch so that gradients reach
the aim offsets; both must give the same numbers.  The derived columns must describe the
heliostat as FieldTracer.aim sets it: the mirror normal of the bisector rule reflects the
sun onto the aim point (east offset, tower height + up offset), seen from the pivot at
HELIO_Z above the field position.
"""
import numpy as np
import torch

from soltrace_b200 import scenes
from soltrace_b200 import surrogate as S


def _situation(n=64, seed=5):
    rng = np.random.default_rng(seed)
    sun, off, sig = S.random_situation(rng, n)
    xy = scenes.field_layout(2000)[rng.choice(2000, n, replace=False)]
    return sun, xy[:, 0].astype(np.float64), xy[:, 1].astype(np.float64), off[:, 0], off[:, 1], sig


def test_numpy_and_torch_features_agree():
    sun, x, y, ox, oy, sig = _situation()
    a = S.situation_features(sun, x, y, ox, oy, sig, 150.0)
    t = S.situation_features(sun, *(torch.as_tensor(v) for v in (x, y, ox, oy)), sig, 150.0, xp=torch)
    assert a.shape == (len(x), S.N_FEATURES) == tuple(t.shape)
    np.testing.assert_allclose(t.numpy(), a, rtol=1e-14, atol=1e-14)


def test_derived_columns_follow_the_bisector_aiming_rule():
    sun, x, y, ox, oy, sig = _situation()
    f = S.situation_features(sun, x, y, ox, oy, sig, 150.0)
    s = np.asarray(sun, dtype=np.float64) / np.linalg.norm(sun)
    np.testing.assert_allclose(f[:, 0:3], np.broadcast_to(s, (len(x), 3)))
    np.testing.assert_allclose(f[:, 3] * 1000.0, x)
    np.testing.assert_allclose(f[:, 4] * 1000.0, y)
    np.testing.assert_allclose(f[:, 5:7], np.stack([ox, oy], 1))
    np.testing.assert_allclose(f[:, 7], sig - 2.0)
    np.testing.assert_allclose(f[:, 8] * 1000.0, np.hypot(x, y))
    np.testing.assert_allclose(np.hypot(f[:, 9], f[:, 10]), 1.0)
    n = f[:, 11:14]
    np.testing.assert_allclose(np.linalg.norm(n, axis=1), 1.0)
    # unit vector from the pivot to the aim point, as FieldTracer.aim builds it
    t = np.stack([ox - x, -y, 150.0 + oy - S.HELIO_Z], 1)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    cos_in = n @ s
    np.testing.assert_allclose(f[:, 14], cos_in)
    np.testing.assert_allclose(f[:, 15], t[:, 2])
    # the sun reflected about the normal goes to the aim point
    refl = 2.0 * cos_in[:, None] * n - s
    np.testing.assert_allclose(refl, t, atol=1e-12)


def test_features_carry_gradients_to_the_aim_offsets():
    sun, x, y, ox, oy, sig = _situation(n=8)
    o = torch.as_tensor(np.stack([ox, oy], 1)).requires_grad_(True)
    f = S.situation_features(sun, torch.as_tensor(x), torch.as_tensor(y), o[:, 0], o[:, 1], sig, 150.0, xp=torch)
    f[:, 11:14].sum().backward()
    g = o.grad.numpy()
    assert np.all(np.isfinite(g)) and np.all(np.abs(g).sum(1) > 0)
