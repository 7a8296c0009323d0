"""The per-ray samplers of the oracle's Philox mode (the same inverse-CDF samplers the
CUDA trace uses) against the reference's rejection samplers, on the CPU.

The oracle's Philox mode restates the device's sampling, so the GPU tests that compare
the device with it ray by ray cannot show that those samplers draw the reference's
distributions.  This test does, without a GPU: the table sunshape 'd' (errors.cpp:160-185)
and the diffuse distribution 'f' (errors.cpp:187-190) through the radial histogram of a
far target, against the reference's results in tests/golden/reference_stats.npz
(tests/golden/make_stat_fixtures.py).  A chi-square p-value below 1e-3 fails.
"""
import dataclasses
import os

import numpy as np
import pytest

from helpers import run_scene
from stat_scenes import rate_z, sampler_scenes, target_radial_from_records, two_sample_chi2

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_stats.npz")
HITS = 400_000


@pytest.mark.parametrize("name", ["sun_table", "diffuse"])
def test_oracle_samplers_match_reference(oracle, name):
    ref = dict(np.load(FIX))
    sc, _, _, rmax, nbins = sampler_scenes()[name]
    sc = dataclasses.replace(sc, raycount=HITS)
    n, rec, _, msg, _ = run_scene(oracle, sc, 23, lambda a, c: a.st_oracle_set_rng(c, 1))
    assert n > 0, msg
    h, on_target = target_radial_from_records(rec, rmax, nbins)
    r_hits, r_on = (int(x) for x in ref[f"{name}_totals"])
    assert abs(rate_z(on_target, HITS, r_on, r_hits)) < 3
    chi2, dof, p = two_sample_chi2(h, HITS, ref[f"{name}_radial"], r_hits)
    assert p > 1e-3, (name, chi2, dof, p)
