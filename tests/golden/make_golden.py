"""Generate tests/golden/reference_runs.json from the reference coretrace.

Run in a checkout where oracle/_ref/coretrace_ref.so has been built from the
reference sources (`make -C oracle ref`):

    python tests/golden/make_golden.py

For every parity scene (tests/scene_zoo.py plus small versions of the dish,
trough and heliostat-field benchmark scenes) the reference's own st_sim_run is
run with a fixed seed, and the fixture keeps the record count, the generated
sun-ray count, the sun box, a sha256 digest of all records in readback order
and the first 32 records verbatim.  The oracle restatement must reproduce the
digests exactly when it replays the reference's random stream.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from soltrace_b200 import scenes  # noqa: E402
from soltrace_b200.capi import StApi  # noqa: E402
from helpers import records_digest, run_scene  # noqa: E402
from scene_zoo import zoo  # noqa: E402

SEED = 11


def golden_scenes(tmpdir: str) -> dict:
    s = dict(zoo(tmpdir))
    s["bench_dish"] = scenes.dish_scene(20000)
    s["bench_trough"] = scenes.trough_scene(20000)
    s["bench_field300"] = scenes.field_scene(300, 20000, dynamic_group=False)
    return s


def main():
    ref = StApi(os.path.join(ROOT, "oracle", "_ref", "coretrace_ref.so"))
    out = {"seed": SEED, "generator": "reference coretrace built from coretrace/*.cpp with g++ -O3", "runs": {}}
    with tempfile.TemporaryDirectory() as td:
        for name, sc in golden_scenes(td).items():
            n, rec, ss, msg, _ = run_scene(ref, sc, SEED)
            entry = {"n": int(n), "sun": ss, "messages": msg}
            if n > 0:
                entry["digest"] = records_digest(rec)
                entry["head"] = {k: [float(v) if k in ("x", "y", "z", "cx", "cy", "cz") else int(v) for v in rec[k][:32]]
                                 for k in rec}
            out["runs"][name] = entry
            print(name, n, ss["nsunrays"])
    with open(os.path.join(HERE, "reference_runs.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
