#!/usr/bin/env python
"""Benchmark of the B200 SolTrace trace.

Metric: ray-stage intersections/s on one B200 for the central-receiver heliostat
field -- 2,000 flat 10x10 m heliostats on a radial-staggered field 100-1000 m north
of a 150 m tower, Buie CSR 0.1 sunshape at 45 deg elevation / 180 deg azimuth,
1.5 mrad slope error, an 8 m x 10 m external cylindrical receiver -- traced to
1e8 first-stage hits per step, in mixed FP32/FP64 precision, with the FP64 device
trace and the flux-map L2 error between them reported beside it.

A step is one st_sim_run of that scene through the C ABI (coretrace_api.so).  A
ray-stage intersection is one generated sun ray or one ray entering a later stage.
`value` divides the units of the K timed steps by their device time (CUDA events on
the library's stream, first launch to last completion); `e2e` divides them by the
wall time of the st_sim_run calls themselves (scene upload from host memory,
kernels, flux and counter readback into host arrays).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) the ranks make one st_sim_run of N x 1e8 hits together
(st_b200_set_ranks: each traces a contiguous slice of every sun-ray batch; one NCCL
all-gather of the ranks' hit counts per batch, one all-reduce of the counters and flux maps
at the end), so the per-GPU work is fixed (weak scaling) and the results equal one GPU's.
`--impl reference` times the reference coretrace (built from its sources into
oracle/_ref/) on the host cores instead.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from soltrace_b200 import flops_model as fm  # noqa: E402
from soltrace_b200 import parallel  # noqa: E402
from soltrace_b200 import scenes  # noqa: E402

METRIC = "ray-stage intersections/s on 1 B200, mixed vs FP64, at <=0.5% flux-map L2 error"
UNIT = "ray-stage intersections/s"
REF_SO = os.path.join(ROOT, "oracle", "_ref", "coretrace_ref.so")
FLUX_MAP = (2, 1, 1, 100, 100, 0.0, 4.0, -5.0, 5.0, 1)  # receiver: 100 x 100 angle x axial, absorbed


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--hits", type=int, default=100_000_000)
    p.add_argument("--helios", type=int, default=2000)
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extra", action="store_true", help="skip the other configurations' lines")
    return p.parse_args()


def workload(args):
    return {"workload": f"heliostat field: {args.helios} flat 10x10 m heliostats, Buie CSR 0.1, "
                        f"8 m x 10 m cylindrical receiver, {args.hits:.0e} first-stage hits per step",
            "heliostats": args.helios, "hits_per_step_per_gpu": args.hits, "receiver_flux_map": "100x100",
            "l2": "per-step working set > L2 (hit lists of up to 0.5 GB per sun-ray batch); "
                  "scene tables (~1 MB) stay L2-resident by design",
            "parallelism": f"dp{args.gpus} (one run's sun-ray range split contiguously over the GPUs)"}


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# reference (CPU) timing
# ---------------------------------------------------------------------------------------
def reference_sample(sc, seconds: float, seed: int):
    """The reference coretrace on all host cores: one context per thread, raycount/threads
    hits each, seeds seed + i*123 (the GUI's multi-thread convention).  Times st_sim_run only."""
    from soltrace_b200.capi import StApi
    if not os.path.exists(REF_SO):
        raise FileNotFoundError(REF_SO)
    ref = StApi(REF_SO)
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    def one(hits, s, out, idx, barrier=None):
        ctx = ref.st_create_context()
        local = dataclasses.replace(sc, raycount=hits, raymax=2_000_000_000 - 1)
        scenes.push(ref, ctx, local)
        if barrier:
            barrier.wait()
        t0 = time.perf_counter()
        n = ref.run(ctx, s)
        dt = time.perf_counter() - t0
        ss = ref.sun_stats(ctx)
        rec = ref.records(ctx)
        ref.st_free_context(ctx)
        entries2 = len(np.unique(rec["raynum"][rec["stage"] == 2])) if n > 0 else 0
        out[idx] = (dt, ss["nsunrays"] + entries2, n)

    # calibrate the per-core rate on a small run
    probe = [None]
    one(2000, seed, probe, 0)
    rate = probe[0][1] / max(probe[0][0], 1e-6)  # units per second per core
    units_per_hit = probe[0][1] / 2000.0
    hits_per_thread = max(2000, int(rate * seconds / units_per_hit))
    res = [None] * ncores
    bar = threading.Barrier(ncores)
    th = [threading.Thread(target=one, args=(hits_per_thread, seed + i * 123, res, i, bar)) for i in range(ncores)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    wall = max(r[0] for r in res)
    units = sum(r[1] for r in res)
    return {"value": units / wall, "unit": UNIT, "cores": ncores, "kind": "reference",
            "sample": f"{ncores} threads x {hits_per_thread} hits ({units} ray-stage units, "
                      f"{wall:.1f} s wall, st_sim_run only, polar receiver hash on)"}


def reference_positions(scene_list, seconds: float, seed: int, label: str):
    """The reference on all host cores, one context per thread, thread i tracing scene
    i % len(scene_list) with seed seed + i*123; hits per thread sized from a calibration run
    so that each thread works about `seconds`.  Times st_sim_run only; returns ray-stage/s."""
    from soltrace_b200.capi import StApi
    if not os.path.exists(REF_SO):
        raise FileNotFoundError(REF_SO)
    ref = StApi(REF_SO)
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    def one(sc, hits, s, out, idx, barrier=None):
        ctx = ref.st_create_context()
        scenes.push(ref, ctx, dataclasses.replace(sc, raycount=hits, raymax=2_000_000_000 - 1))
        if barrier:
            barrier.wait()
        t0 = time.perf_counter()
        n = ref.run(ctx, s)
        dt = time.perf_counter() - t0
        if n < 0:
            raise RuntimeError("reference st_sim_run failed: " + "; ".join(ref.messages(ctx)))
        ss = ref.sun_stats(ctx)
        rec = ref.records(ctx)
        ref.st_free_context(ctx)
        later = sum(len(np.unique(rec["raynum"][rec["stage"] == k])) for k in range(2, 17)) if n > 0 else 0
        out[idx] = (dt, ss["nsunrays"] + later, n)

    probe = [None]
    one(scene_list[0], 500, seed, probe, 0)
    rate = probe[0][1] / max(probe[0][0], 1e-6)
    hits_per_thread = max(500, int(rate * seconds / max(probe[0][1] / 500.0, 1e-9)))
    res = [None] * ncores
    bar = threading.Barrier(ncores)
    th = [threading.Thread(target=one, args=(scene_list[i % len(scene_list)], hits_per_thread, seed + i * 123, res, i,
                                             bar)) for i in range(ncores)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    wall = max(r[0] for r in res)
    units = sum(r[1] for r in res)
    return {"value": units / wall, "unit": UNIT, "cores": ncores, "kind": "reference",
            "sample": f"{label}: {ncores} threads x {hits_per_thread} hits ({units} ray-stage units, {wall:.1f} s wall, "
                      "st_sim_run only)"}


def config_lines(api, args) -> dict:
    """The other benchmark configurations, each timed beside the reference on the host cores:
    C1 dish (FP64, 1e6 hits, 50 x 50 absorber map), C2 trough (FP64 and mixed, 1e7 hits,
    72 x 120 absorber-tube map), C4 batched annual beam-down trace (512 sun positions, tracking
    field of 10,000 heliostats, 64 x 64 ground map, one st_b200_sim_run_batch call), the
    headline field with records on (1e7 hits, st_locations & co. read back: what pysoltrace
    pays), and the C5 flux surrogate."""
    out = {}

    def timed_runs(sc, maps, prec, seed, steps, records=False):
        ctx = api.st_create_context()
        scenes.push(api, ctx, sc)
        api.st_b200_set_precision(ctx, prec)
        api.st_b200_set_records(ctx, 1 if records else 0)
        for m in maps:
            api.st_b200_add_flux_map(ctx, *m)
        for w in range(3):  # warm-up: scene set-up, autotuning, buffers sized for the planned batches
            api.run(ctx, seed + 1000 + w)
        units = dev = wall = 0.0
        flux = None
        for k in range(steps):
            t0 = time.perf_counter()
            rc = api.run(ctx, seed + 1 + k)
            if records and rc > 0:
                api.records(ctx)
            wall += time.perf_counter() - t0
            if rc < 0:
                raise RuntimeError("; ".join(api.messages(ctx)))
            st = api.stats(ctx)
            units += st["ray_stage_units"]
            dev += st["kernel_ms"] / 1e3
            flux = [api.flux(ctx, i, m[3], m[4]) for i, m in enumerate(maps)]
        api.st_free_context(ctx)
        return {"value": units / dev, "e2e": units / wall, "ms_per_step": dev / steps * 1e3,
                "units_per_step": units / steps}, flux

    seconds = min(args.cpu_seconds, 8.0)
    # C1: dish
    dish = scenes.dish_scene(1_000_000)
    c1, _ = timed_runs(dish, [(2, 1, 0, 50, 50, -0.25, 0.25, -0.25, 0.25, 1)], 0, 1, 3)
    c1.update(workload="C1 parabolic dish + flat absorber, pillbox sun, 1e6 hits, 50x50 map", dtype="f64")
    # C2: trough, FP64 and mixed
    trough = scenes.trough_scene(10_000_000)
    tmap = [(3, 2, 1, 72, 120, 0.0, 0.035, -6.0, 6.0, 1)]
    c2, f64 = timed_runs(trough, tmap, 0, 2, 2)
    c2m, fmx = timed_runs(trough, tmap, 1, 2, 2)
    a, b = f64[0].astype(float), fmx[0].astype(float)
    c2.update(workload="C2 parabolic trough + glass envelope + absorber tube, gaussian sun, 1e7 hits, 72x120 map",
              dtype="f64", mixed={"value": c2m["value"], "ms_per_step": c2m["ms_per_step"],
                                  "flux_l2_mixed_vs_fp64": float(np.linalg.norm(a - b) / max(np.linalg.norm(a), 1e-30))})
    # headline field with records (pysoltrace's path)
    fld = scenes.field_scene(args.helios, 10_000_000)
    rec, _ = timed_runs(fld, [FLUX_MAP], 1, 5, 2, records=True)
    rec.update(workload="C3 field, 1e7 hits, records on and read back (st_locations, st_cosines, st_elementmap, "
                        "st_stagemap, st_raynumbers)", dtype="fp32+fp64 (mixed)")
    out["records_on_field_1e7"] = rec
    # C4: batched annual beam-down trace
    suns, hits, dni = scenes.annual_suns(512)
    bd = scenes.beam_down_scene(10_000, raycount=1000)
    ctx = api.st_create_context()
    scenes.push(api, ctx, bd)
    api.st_b200_set_precision(ctx, 1)
    api.st_b200_add_flux_map(ctx, *scenes.GROUND_MAP)
    tgt = scenes.beam_down_target()
    # warm-up: two full chunks (128 positions spread over the year, a tenth of their hits), so
    # the timed call finds its device buffers and both page-locked staging areas already sized
    api.run_batch(ctx, 100, suns[::4], hits[::4] // 10, tgt)
    t0 = time.perf_counter()
    rc = api.run_batch(ctx, 100, suns, hits, tgt)
    wall = time.perf_counter() - t0
    if rc < 0:
        raise RuntimeError("; ".join(api.messages(ctx)))
    tot = api.batch_stats(ctx, -1)
    intercept = []
    for k in range(len(hits)):
        g = api.batch_flux(ctx, 0, k, scenes.GROUND_MAP[3], scenes.GROUND_MAP[4])
        intercept.append(float(g.sum()) / max(hits[k], 1))
    api.st_free_context(ctx)
    c4 = {"value": tot["ray_stage_units"] / (tot["kernel_ms"] / 1e3), "e2e": tot["ray_stage_units"] / wall,
          "unit": UNIT, "positions": len(hits), "hits": int(hits.sum()), "sun_rays": tot["sun_rays"],
          "device_ms": tot["kernel_ms"], "wall_ms": wall * 1e3, "host_setup_ms": tot["setup_ms"],
          "gpu_launches": tot["gpu_launches"], "h2d_bytes": tot["h2d_bytes"],
          "mean_ground_intercept_per_hit": float(np.mean(intercept)), "dtype": "fp32+fp64 (mixed)",
          "workload": "C4 beam-down: 10,000 tracking heliostats, hyperboloid secondary (e 1.3) with torus lip, "
                      "64x64 ground receiver; 512 sun positions at 40 N, 1e6 x DNI/1000 hits each"}
    if not args.no_cpu_baseline:
        for name, line, sc_list in (("C1", c1, [dish]), ("C2", c2, [trough]),
                                    ("C4", c4, [scenes.beam_down_scene(10_000, raycount=1000, sun_xyz=suns[k])
                                                for k in range(16)])):
            try:
                line["reference"] = reference_positions(sc_list, seconds, 7, name)
                line["vs_reference"] = line["value"] / line["reference"]["value"]
            except Exception as ex:  # noqa: BLE001
                line["reference"] = {"unavailable": str(ex)}
    out["C1_dish"], out["C2_trough"], out["C4_batch"] = c1, c2, c4
    try:  # a failure here keeps the lines above
        out["C5_surrogate"] = surrogate_line(api)
    except Exception as ex:  # noqa: BLE001
        out["C5_surrogate"] = {"error": str(ex)}
    return out


# 20,000 Adam steps with the rate decayed 2e-3 -> 6e-5: on the same data, 16 held-out peak
# errors of max 2.1 % (mean 1.0 %) against 3.1 % (1.3 %) for 12,000 steps decayed 2e-3 -> 2e-4
N_TRAIN_TRACES, N_TRAIN_STEPS, N_TRAIN_BATCH, N_TRAIN_LR_FINAL = 1000, 20000, 16384, 0.03


def surrogate_line(api) -> dict:
    """C5: the BF16 flux surrogate (6 layers, width 256, 32 x 32 receiver image per heliostat)
    trained on the device from 2e6 traced samples (1,000 traces of the headline field at 1e7
    hits, each giving 2,000 per-heliostat images), compared on 16 held-out situations traced at
    1e7 hits, and timed predicting the field maps of 64 sun positions x 2,000 heliostats in one
    fused pass against the plain trace of one position at 1e7 hits."""
    import torch

    from soltrace_b200 import surrogate as S
    tracer = S.FieldTracer(api)
    try:
        net, scale, t_data, t_train = S.fit(tracer, N_TRAIN_TRACES, 10_000_000, N_TRAIN_STEPS, batch=N_TRAIN_BATCH,
                                            lr_final=N_TRAIN_LR_FINAL)
        noise = []
        peaks, l1 = S.evaluate(net, tracer, scale, 16, 10_000_000, noise=noise)
        untrained = S.Mlp(api, seed=77)
        peaks0, l10 = S.evaluate(untrained, tracer, scale, 4, 10_000_000)
        ms = S.time_fields(net, tracer, scale, n_suns=64)
        rng = np.random.default_rng(5)
        trace_ms = []
        for i in range(4):
            tracer.trace(*S.random_situation(rng, tracer.n), 10_000_000, 900 + i)
            trace_ms.append(api.stats(tracer.ctx)["kernel_ms"])
        assert net.error() == 0
    finally:
        tracer.close()
    peaks_file = os.path.join(ROOT, "MEASURED_PEAKS.json")
    bf16 = None
    if os.path.exists(peaks_file):
        bf16 = json.load(open(peaks_file)).get("bf16_tflops")
    flops = S.fused_flops(S.DIMS, 64 * 2000)
    tflops = flops / (ms / 1e3) / 1e12
    per_trace = float(np.median(trace_ms))
    return {"workload": "C5 BF16 MLP flux surrogate (16 -> 5 x 256 -> 1024), field maps of 64 suns x 2,000 "
                        "heliostats in one fused tcgen05 pass vs the trace of one sun at 1e7 hits",
            "speedup": 64 * per_trace / ms, "surrogate_ms_64_suns": ms, "trace_ms_per_sun_1e7": per_trace,
            "peak_error_max": max(peaks), "peak_error_mean": float(np.mean(peaks)),
            "trace_repeat_peak_error_max": max(noise), "trace_repeat_peak_error_mean": float(np.mean(noise)),
            "map_l1_error_mean": float(np.mean(l1)), "untrained_peak_error_mean": float(np.mean(peaks0)),
            "untrained_map_l1_error_mean": float(np.mean(l10)), "train_traces": N_TRAIN_TRACES,
            "train_samples": N_TRAIN_TRACES * 2000, "train_steps": N_TRAIN_STEPS, "train_batch": N_TRAIN_BATCH,
            "trace_data_s": t_data, "train_s": t_train, "dtype": "bf16 (fp32 accumulate)",
            "roofline": {"bound": "tensor", "kernel": "k_mlp_fused", "achieved": tflops,
                         "peak": bf16, "unit": "TFLOP/s", "frac": tflops / bf16 if bf16 else None,
                         "peak_source": "of measured (bf16 burst)" if bf16 else "unavailable"}}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc = scenes.field_scene(args.helios, args.hits)
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/coretrace_ref.so not built"}))
        return
    per_step = max(2.0, min(args.cpu_seconds, 20.0))
    vals = []
    for k in range(args.warmup + args.steps):
        r = reference_sample(sc, per_step, args.seed + k)
        if k >= args.warmup:
            vals.append(r)
    value = statistics.median([v["value"] for v in vals])
    cb = dict(vals[-1])
    cb["value"] = value
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload(args),
            "cpu_baseline": cb, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# B200 arm
# ---------------------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import torch

    from soltrace_b200.lib import load
    api = load()
    # weak scaling: the run numbers args.hits first-stage hits per GPU; over N GPUs it is one
    # st_sim_run of N x args.hits hits split over the ranks (st_b200_set_ranks), with the
    # results of that run on one GPU
    sc = scenes.field_scene(args.helios, args.hits * world)
    ctx = api.st_create_context()
    scenes.push(api, ctx, sc)
    api.st_b200_set_device(ctx, local if world > 1 else 0)
    api.st_b200_set_records(ctx, 0)
    api.st_b200_add_flux_map(ctx, *FLUX_MAP)
    if api.has("st_b200_set_max_sun_rays"):
        api.st_b200_set_max_sun_rays(ctx, 40 * args.hits * world)  # beyond st_sim_params' int cap
    exchange = None
    if world > 1:
        exchange = parallel.RankExchange(device="cuda")
        if exchange.attach(api, ctx) != 1:
            raise RuntimeError("st_b200_set_ranks failed: " + "; ".join(api.messages(ctx)))

    def step(prec, seed):
        api.st_b200_set_precision(ctx, prec)
        t0 = time.perf_counter()
        rc = api.run(ctx, seed)
        wall = time.perf_counter() - t0
        if rc < 0:
            raise RuntimeError("st_sim_run failed: " + "; ".join(api.messages(ctx)))
        st = api.stats(ctx)
        st["wall_ms"] = wall * 1e3
        st["flux"] = api.flux(ctx, 0, FLUX_MAP[3], FLUX_MAP[4])
        return st

    seed0 = args.seed  # every rank runs the same seed: the ranks share one run
    for k in range(args.warmup):
        step(1, seed0 + k)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    runs = []
    with ClockSampler(local) as clk:
        barrier()
        for k in range(args.steps):
            runs.append(step(1, seed0 + 100 + k))
        barrier()
    units = sum(r["ray_stage_units"] for r in runs)
    dev_ms = sum(r["kernel_ms"] for r in runs)
    wall_ms = sum(r["wall_ms"] for r in runs)
    probe_ms = sum(r["probe_ms"] for r in runs)
    trace_ms = sum(r["trace_ms"] for r in runs)
    launches = sum(r["gpu_launches"] for r in runs)

    # FP64 device trace of the same steps: throughput and the flux-map L2 error
    n64 = max(1, min(args.steps, 2))
    for k in range(max(1, min(args.warmup, 3))):  # untimed, as for the mixed steps
        step(0, seed0 + k)
    runs64 = [step(0, seed0 + 100 + k) for k in range(n64)]
    units64 = sum(r["ray_stage_units"] for r in runs64)
    dev64 = sum(r["kernel_ms"] for r in runs64)
    l2 = [float(np.linalg.norm(runs[k]["flux"].astype(float) - runs64[k]["flux"].astype(float)) /
                max(np.linalg.norm(runs64[k]["flux"].astype(float)), 1e-30)) for k in range(n64)]

    # whole-job totals: the units are the run's (already over all ranks), device and wall
    # times the max over ranks
    units, dev_ms, wall_ms = parallel.combine(units, dev_ms, wall_ms, device="cuda" if dist else "cpu")
    flux_sum = runs[-1]["flux"]
    if rank != 0:
        api.st_free_context(ctx)
        if dist:
            dist.destroy_process_group()
        return

    value = units / (dev_ms / 1e3)
    e2e = units / (wall_ms / 1e3)
    last = runs[-1]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    sun_rays = sum(r["sun_rays"] for r in runs)
    hits = sum(r["ray_hits"] for r in runs)
    rec_entries = sum(r["stage_entries"][1] for r in runs)
    pf, tf = fm.probe_flops(sun_rays), fm.trace_flops(hits, rec_entries)
    probe_tflops = pf / (probe_ms / 1e3) / 1e12
    trace_tflops = tf / (trace_ms / 1e3) / 1e12
    dominant = "k_probe" if probe_ms >= trace_ms else "k_trace"
    # DRAM bytes per unit of each launch group (ncu captures at 2e6 hits), scaled to this
    # step's units
    if dominant == "k_probe":
        traffic = fm.DRAM_BYTES_PER_SUN_RAY_PROBE * sun_rays / len(runs)
    else:
        traffic = fm.DRAM_BYTES_PER_HIT_TRACE * hits / len(runs)
    if dominant == "k_probe":
        ach, pk = probe_tflops, fm.NOMINAL_FP64_TFLOPS
        hbm_ach = fm.probe_bytes(sun_rays, hits) / (probe_ms / 1e3) / 1e9
    else:
        ach, pk = trace_tflops, fm.NOMINAL_FP64_TFLOPS
        hbm_ach = fm.trace_bytes(hits) / (trace_ms / 1e3) / 1e9
    clk_summary = clk.summary()
    clk_mhz = clk_summary.get("sm_mhz") or 1965.0
    issue_peak = fm.issue_peak_per_s(clk_mhz)
    group = {"k_probe": "probe group (k_sun_probe_exact or k_sun_candidates + k_sun_resolve, block-count scan, "
                        "element sort)",
             "k_trace": "trace group (k_wf_first, k_wf_search, k_wf_shade, k_wf_finish)"}[dominant]
    roofline = {"bound": "fp64", "kernel": group, "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "scope": "per step: the group's launches of every batch, timed by CUDA events around them",
                "traffic_unit": "DRAM bytes per step (ncu per-unit figures scaled)",
                "frac": ach / pk, "peak_source": "nominal (148 SMs x 64 FP64 lanes x 2 x 1965 MHz); "
                                                 "no measured FP64 vector peak on this pool",
                "traffic": traffic,
                "hbm": {"achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_ach / hbm_peak,
                        "peak_source": "of measured" if "hbm_gbs" in peaks else "of fallback"},
                "split_ms_per_step": {"k_probe+compact": probe_ms / len(runs), "k_trace": trace_ms / len(runs)},
                "probe_tflops": probe_tflops, "trace_tflops": trace_tflops,
                # instruction issue: warp instructions per unit (ncu, flops_model) x units / the
                # group's device time, against four warp instructions per SM and cycle
                "issue": {
                    "unit": "warp instructions/s",
                    "peak": issue_peak,
                    "peak_source": f"148 SMs x 4 schedulers x {clk_mhz:.0f} MHz (median SM clock of the timed steps)",
                    "probe_group_frac": fm.WARP_INSTR_PER_SUN_RAY_PROBE * sun_rays / (probe_ms / 1e3) / issue_peak,
                    "trace_group_frac": fm.WARP_INSTR_PER_HIT_TRACE * hits / (trace_ms / 1e3) / issue_peak}}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            cpu = reference_sample(scenes.field_scene(args.helios, args.hits), args.cpu_seconds, args.seed)
        except Exception as ex:  # noqa: BLE001
            cpu = {"value": None, "unavailable": str(ex)}

    extra = None
    if world == 1 and not args.no_extra:
        try:
            extra = config_lines(api, args)
        except Exception as ex:  # noqa: BLE001
            extra = {"error": str(ex)}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / len(runs), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32+fp64 (mixed)", "data": "synthetic (seeded heliostat layout and aim jitter)",
        "config": workload(args),
        "fp64": {"value": units64 / (dev64 / 1e3), "ms_per_step": dev64 / n64,
                 "mixed_speedup": value / (units64 / (dev64 / 1e3)), "flux_l2_mixed_vs_fp64": max(l2)},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(last["h2d_bytes"]),
                "d2h_bytes_per_step": int(last["d2h_bytes"]), "ms_per_step": wall_ms / len(runs)},
        "gpu_launches": int(launches),
        "autotuned_variants": {"probe": runs[-1]["probe_variant"], "trace": runs[-1]["trace_variant"],
                               "fp64_trace": runs64[-1]["trace_variant"]},
        "units_per_step": units / len(runs), "sun_rays_per_step": sun_rays / len(runs),
        "receiver_flux_counts": int(flux_sum.sum()),
        "roofline": roofline, "clocks": clk_summary, "cpu_baseline": cpu,
        "other_configs": extra,
    }
    print(json.dumps(line), flush=True)
    api.st_free_context(ctx)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
