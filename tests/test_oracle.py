"""The CPU oracle against the reference (no GPU needed).

The oracle restates coretrace's trace; replaying the reference's libstdc++
random stream it must reproduce the reference's records bit for bit.  The
golden fixture (tests/golden/reference_runs.json, made by
tests/golden/make_golden.py from the reference built from its own sources)
pins it on every parity scene; when the reference library is present the same
comparison also runs live on other seeds.
"""
import json
import os

import numpy as np
import pytest

from helpers import records_digest, run_scene
from soltrace_b200 import scenes

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_runs.json")))


def _golden_scenes(zoo_scenes):
    s = dict(zoo_scenes)
    s["bench_dish"] = scenes.dish_scene(20000)
    s["bench_trough"] = scenes.trough_scene(20000)
    s["bench_field300"] = scenes.field_scene(300, 20000, dynamic_group=False)
    return s


@pytest.mark.parametrize("name", sorted(GOLDEN["runs"]))
def test_oracle_reproduces_reference_golden(oracle, zoo_scenes, name):
    sc = _golden_scenes(zoo_scenes)[name]
    g = GOLDEN["runs"][name]
    n, rec, ss, msg, _ = run_scene(oracle, sc, GOLDEN["seed"], lambda a, c: a.st_oracle_set_rng(c, 0))
    assert n == g["n"], msg
    assert ss["nsunrays"] == g["sun"]["nsunrays"]
    for k in ("xmin", "xmax", "ymin", "ymax"):
        assert ss[k] == g["sun"][k]
    if n > 0:
        assert records_digest(rec) == g["digest"]
        for k, v in g["head"].items():
            np.testing.assert_array_equal(rec[k][: len(v)], np.asarray(v, dtype=rec[k].dtype))
    else:
        assert msg == g["messages"]


@pytest.mark.parametrize("name,seed", [("dish", 3), ("trough", 5), ("refraction", 7), ("spline", 9), ("torus", 13),
                                       ("fe_surface", 15)])
def test_oracle_matches_live_reference(oracle, reference, zoo_scenes, name, seed):
    if name == "dish":
        sc = scenes.dish_scene(5000)
    elif name == "trough":
        sc = scenes.trough_scene(5000)
    else:
        sc = zoo_scenes[name]
    a = run_scene(reference, sc, seed)
    b = run_scene(oracle, sc, seed, lambda x, c: x.st_oracle_set_rng(c, 0))
    assert a[0] == b[0] and a[2] == b[2]
    assert records_digest(a[1]) == records_digest(b[1])


def test_oracle_dynamic_group_field(oracle, reference):
    """Heliostat field with the reference's polar receiver hash switched on: on this
    layout it culls nothing the brute-force search would find."""
    sc = scenes.field_scene(120, 3000, dynamic_group=True)
    a = run_scene(reference, sc, 3)
    b = run_scene(oracle, sc, 3, lambda x, c: x.st_oracle_set_rng(c, 0))
    assert a[0] == b[0] and records_digest(a[1]) == records_digest(b[1])


def test_oracle_errors_match_reference_messages(oracle, reference):
    """Failure paths return -1 with the reference's message."""
    bad = scenes.dish_scene(100)
    bad.stages[0].elements[0].optic = "no-such-optic"
    for api in (oracle, reference):
        n, _, _, msg, _ = run_scene(api, bad, 1)
        assert n == -1 and "invalid optical property set name" in msg[0]
    tight = scenes.dish_scene(1000)
    tight.raymax = 500
    ra = run_scene(reference, tight, 1)
    rb = run_scene(oracle, tight, 1)
    assert ra[0] == rb[0] == -1 and ra[3] == rb[3]


def test_oracle_philox_stream_is_per_ray(oracle):
    """With the per-ray stream, a ray's records do not depend on how many rays are traced."""
    small = scenes.dish_scene(200)
    big = scenes.dish_scene(400)
    a = run_scene(oracle, small, 5, lambda x, c: x.st_oracle_set_rng(c, 1))
    b = run_scene(oracle, big, 5, lambda x, c: x.st_oracle_set_rng(c, 1))
    ra, rb = a[1], b[1]
    for s in (1, 2):
        ma = (ra["stage"] == s)
        mb = (rb["stage"] == s) & (rb["raynum"] <= 200)
        for k in ("x", "y", "z", "element", "raynum"):
            np.testing.assert_array_equal(np.sort(ra[k][ma]), np.sort(rb[k][mb]))


@pytest.mark.parametrize("sun_elev_az", [None, (30.0, 120.0)])
def test_oracle_matches_reference_on_beam_down(oracle, reference, sun_elev_az):
    """The batched study's geometry (heliostats aimed at the upper focus of a convex
    hyperboloid secondary with an absorbing torus lip, ground receiver under the lower focus),
    at 300 heliostats: records bit for bit, with rays on the lip and on the ground."""
    sun = None if sun_elev_az is None else scenes.sun_vector(*sun_elev_az)
    sc = scenes.beam_down_scene(300, raycount=3000, sun_xyz=sun)
    a = run_scene(reference, sc, 5)
    b = run_scene(oracle, sc, 5, lambda x, c: x.st_oracle_set_rng(c, 0))
    assert a[0] == b[0] > 0 and a[2] == b[2]
    assert records_digest(a[1]) == records_digest(b[1])
    rec = a[1]
    assert np.sum((rec["stage"] == 2) & (np.abs(rec["element"]) == 2)) > 0  # the torus lip
    assert np.sum((rec["stage"] == 3) & (rec["element"] < 0)) > 0           # absorbed on the ground
