"""Generate tests/golden/reference_stats.npz: statistical-mode results of the reference.

Run in a checkout where oracle/_ref/coretrace_ref.so has been built from the reference
sources (`make -C oracle ref`):

    python tests/golden/make_stat_fixtures.py

The reference's own st_sim_run traces each scene on all host cores, one context per
thread with an equal share of the hits (the GUI's multi-thread convention,
app/src/trace.cpp:709-728), each thread seeded at an evenly spaced point of the
generator's cycle (stat_scenes.spaced_seeds) so that no two threads draw the same random
numbers.  From its records this script keeps what the statistical parity tests compare
against the CUDA trace (tests/test_gpu_statistics.py) and the oracle's per-ray sampler
(tests/test_oracle_statistics.py):

* "field" (Buie CSR 0.1 table sunshape, the headline configuration, 4e6 first-stage hits: the
  most the reference's generator cycle holds without repeating its random numbers, see
  stat_scenes.REFERENCE_HITS) and "field_gauss" (the same field under a 2.73 mrad Gaussian
  sun, 1e7 hits): the central-receiver heliostat field (2,000 flat heliostats, cylindrical
  receiver) with exact culling
  (include_dynamic_group = 0): the 100 x 100 receiver flux map of absorbed rays, binned by
  pysoltrace's cylinder rule (app/deploy/api/pysoltrace.py:1896-1942), the per-heliostat
  first hits and deliveries (rays absorbed on the receiver, joined to their first
  heliostat by ray number), and the run totals;
* "sun_table": a flat mirror under the same table sunshape, reflecting onto a far target:
  the radial histogram of target hits measures the sampled sun angles (errors.cpp:160-185);
* "diffuse": a flat mirror with the diffuse optical distribution 'f' (errors.cpp:187-190)
  under a near-collimated sun: the radial histogram on a wide target above it;
* "theta": 4e6 sun angles drawn by the reference's table-sunshape sampler (a 0.2 mm mirror
  under the Buie table, onto a target 500 m away), histogrammed in mrad; the tests compare
  it, and the oracle's sampler, with the distribution the table defines.
"""
from __future__ import annotations

import dataclasses
import json
import math
import os
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from soltrace_b200.capi import StApi  # noqa: E402
from stat_scenes import (FIELD_FLUX, REFERENCE_HITS, field_stat_scene, sampler_scenes, spaced_seeds,  # noqa: E402
                         receiver_flux_from_records, per_heliostat_from_records, target_radial_from_records,
                         sun_theta_scene, theta_histogram)

OUT = os.path.join(HERE, "reference_stats.npz")


def traced(ref: StApi, sc, hits_total: int, seed: int, threads: int):
    """Records of `threads` contexts of the reference, each tracing hits_total/threads hits
    (remainder to the first), seeded by spaced_seeds(threads, seed).  Returns a list of
    (records, sun stats)."""
    share = [hits_total // threads] * threads
    share[0] += hits_total - sum(share)
    seeds = spaced_seeds(threads, seed)
    out = [None] * threads

    def one(i):
        ctx = ref.st_create_context()
        from soltrace_b200 import scenes
        scenes.push(ref, ctx, dataclasses.replace(sc, raycount=share[i]))
        n = ref.run(ctx, seeds[i])
        if n < 0:
            raise RuntimeError(ref.messages(ctx))
        out[i] = (ref.records(ctx), ref.sun_stats(ctx))
        ref.st_free_context(ctx)

    th = [threading.Thread(target=one, args=(i,)) for i in range(threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return out


def main():
    ref = StApi(os.path.join(ROOT, "oracle", "_ref", "coretrace_ref.so"))
    threads = len(os.sched_getaffinity(0))
    arrays, meta = {}, {"generator": "reference coretrace built from coretrace/*.cpp with g++ -O3",
                        "threads": threads, "seed_rule": "stat_scenes.spaced_seeds(threads, seed)"}

    for key, sun in (("field", "buie"), ("field_gauss", "gauss")):
        t0 = time.time()
        sc, _, seed = field_stat_scene(sun)
        hits = REFERENCE_HITS[sun]
        runs = traced(ref, sc, hits, seed, threads)
        flux = np.zeros((FIELD_FLUX[4], FIELD_FLUX[3]), dtype=np.int64)
        n_el = len(sc.stages[0].elements)
        first = np.zeros(n_el, dtype=np.int64)
        delivered = np.zeros(n_el, dtype=np.int64)
        sun_rays = 0
        for rec, ss in runs:
            flux += receiver_flux_from_records(ref, sc, rec)
            f, d = per_heliostat_from_records(rec, n_el)
            first += f
            delivered += d
            sun_rays += int(ss["nsunrays"])
        arrays.update({f"{key}_flux": flux, f"{key}_first": first, f"{key}_delivered": delivered,
                       f"{key}_totals": np.array([hits, sun_rays, int(flux.sum())], dtype=np.int64)})
        meta[key] = {"hits": hits, "seed": seed, "sun": sun, "sun_rays": sun_rays,
                     "absorbed_on_receiver": int(flux.sum()), "seconds": round(time.time() - t0, 1)}
        print(key, meta[key], flush=True)

    t0 = time.time()
    hits = 4_000_000
    runs = traced(ref, sun_theta_scene(hits), hits, 31, threads)
    arrays["theta"] = sum(theta_histogram(rec) for rec, _ in runs)
    meta["theta"] = {"hits": hits, "seed": 31, "seconds": round(time.time() - t0, 1)}
    print("theta", meta["theta"], flush=True)

    for name, (sc, hits, seed, rmax, nbins) in sampler_scenes().items():
        t0 = time.time()
        runs = traced(ref, sc, hits, seed, threads)
        h = np.zeros(nbins, dtype=np.int64)
        absorbed = 0
        for rec, _ in runs:
            hh, a = target_radial_from_records(rec, rmax, nbins)
            h += hh
            absorbed += a
        arrays[f"{name}_radial"] = h
        arrays[f"{name}_totals"] = np.array([hits, absorbed], dtype=np.int64)
        meta[name] = {"hits": hits, "seed": seed, "on_target": absorbed, "edges_m": [0.0, rmax], "bins": nbins,
                      "seconds": round(time.time() - t0, 1)}
        print(name, meta[name], flush=True)

    np.savez_compressed(OUT, **arrays)
    with open(OUT.replace(".npz", ".json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
