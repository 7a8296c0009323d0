"""First stages with more elements than the shared-memory counting sort has bins (11,264)
sort the probe's hits with global atomics instead (k_list_hist, k_list_scatter), which also
hand out the ray numbers.  A 12,000-heliostat field must still trace ray by ray as the
oracle does: same ray numbers, elements and SunRayCount, positions within 1e-9 m.
"""
import numpy as np
import pytest

from helpers import assert_same_records, run_scene
from soltrace_b200 import scenes

pytestmark = pytest.mark.gpu


def test_large_first_stage_matches_oracle(product, oracle):
    sc = scenes.field_scene(12000, 3000, dynamic_group=False)
    assert len(sc.stages[0].elements) > 11264
    a = run_scene(product, sc, 7, lambda api, ctx: api.st_b200_set_precision(ctx, 0))
    b = run_scene(oracle, sc, 7, lambda api, ctx: api.st_oracle_set_rng(ctx, 1))
    assert a[0] == b[0] > 0, (a[3], b[3])
    assert a[2] == b[2]  # sun box and SunRayCount (the cut-off at the 3,000th hit)
    first = a[1]["raynum"][a[1]["stage"] == 1]
    np.testing.assert_array_equal(np.unique(first), np.arange(1, 3001))
    assert_same_records(a[1], b[1], pos_tol=1e-9, rel_tol=2e-12, dir_tol=1e-9)
