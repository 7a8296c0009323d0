"""Geometry of the beam-down scene (no GPU): the secondary's foci and aiming rule.

scenes.beam_down_geometry gives the convex hyperboloid secondary (SolTrace surface 'o':
x^2 + y^2 + kappa z^2 - 2 z / c = 0, vertex at BEAM_DOWN_HEIGHT) and the heights of its two
foci.  A ray travelling toward the upper focus must leave the mirror toward the lower focus
(the reflective property the beam-down design relies on), the upper focus must sit
FOCUS_BELOW_RIM under the rim plane so that rays aimed at it meet the mirror, and the
tracking target the batched runs use is that focus.
"""
import math

import numpy as np

from soltrace_b200 import scenes


def test_rays_toward_the_upper_focus_reflect_toward_the_lower_focus():
    c, kappa, f1, f2 = scenes.beam_down_geometry()
    h = scenes.BEAM_DOWN_HEIGHT
    R = 1.0 / c
    assert math.isclose(kappa, 1.0 - scenes.BEAM_DOWN_ECC ** 2)
    assert f2 < h < f1
    F1, F2 = np.array([0.0, 0.0, f1]), np.array([0.0, 0.0, f2])
    for r in np.linspace(0.5, scenes.BEAM_DOWN_DIAM / 2.0 - 0.1, 12):
        for phi in (0.0, 1.1, 2.5):
            z = scenes._hyperboloid_sag(R, kappa, r)
            x, y = r * math.cos(phi), r * math.sin(phi)
            assert abs(x * x + y * y + kappa * z * z - 2.0 * z * R) < 1e-9 * R * R
            P = np.array([x, y, h + z])
            n = np.array([2.0 * x, 2.0 * y, 2.0 * kappa * z - 2.0 * R])
            n /= np.linalg.norm(n)
            d = (F1 - P) / np.linalg.norm(F1 - P)
            out = d - 2.0 * np.dot(d, n) * n
            to_f2 = (F2 - P) / np.linalg.norm(F2 - P)
            assert np.dot(out, to_f2) > 1.0 - 1e-12, (r, phi)


def test_upper_focus_under_the_rim_and_tracking_target():
    c, kappa, f1, _ = scenes.beam_down_geometry()
    rim = scenes.BEAM_DOWN_HEIGHT + scenes._hyperboloid_sag(1.0 / c, kappa, scenes.BEAM_DOWN_DIAM / 2.0)
    assert abs((rim - f1) - scenes.FOCUS_BELOW_RIM) < 1e-9
    np.testing.assert_array_equal(scenes.beam_down_target(), [0.0, 0.0, f1])
