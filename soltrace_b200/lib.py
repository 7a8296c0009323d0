"""Loader for the in-tree coretrace_api.so (the CUDA product).

`load()` returns a `StApi` bound to soltrace_b200/coretrace_api.so with the
st_b200_* extension signatures added.  It raises if the library has not been
built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .capi import StApi, c_double_p, st_uint_t

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "coretrace_api.so")

ST_B200_FP64 = 0
ST_B200_MIXED = 1


class Stats(C.Structure):
    _fields_ = [
        ("sun_rays", C.c_ulonglong),
        ("ray_hits", C.c_ulonglong),
        ("stage_entries", C.c_ulonglong * 16),
        ("ray_stage_units", C.c_ulonglong),
        ("records", C.c_ulonglong),
        ("kernel_ms", C.c_double),
        ("probe_ms", C.c_double),
        ("trace_ms", C.c_double),
        ("setup_ms", C.c_double),
        ("readback_ms", C.c_double),
        ("batches", C.c_int),
        ("gpu_launches", C.c_int),
        ("h2d_bytes", C.c_ulonglong),
        ("d2h_bytes", C.c_ulonglong),
        ("probe_variant", C.c_int),
        ("trace_variant", C.c_int),
        ("intersections", C.c_ulonglong),
    ]


class FluxStats(C.Structure):
    """st_b200_flux_stats_t: the GUI's element flux statistics of one flux map."""
    _fields_ = [(k, C.c_double) for k in ("peak_flux", "min_flux", "ave_flux", "sigma_flux", "uniformity",
                                          "peak_flux_uncertainty", "ave_flux_uncertainty", "power_per_ray",
                                          "bin_area")] + \
               [(k, C.c_ulonglong) for k in ("rays_binned", "rays_in_peak_bin", "rays_in_min_bin")]


_u64p = C.POINTER(C.c_ulonglong)
EXTENSIONS = {
    "st_b200_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "st_b200_set_records": (C.c_int, [C.c_void_p, C.c_int]),
    "st_b200_set_device": (C.c_int, [C.c_void_p, C.c_int]),
    "st_b200_explicit_rays": (C.c_int, [C.c_void_p, st_uint_t, c_double_p, c_double_p]),
    "st_b200_add_flux_map": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_int]),
    "st_b200_add_source_flux_map": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                              C.c_double, C.c_double, C.c_double, C.c_int]),
    "st_b200_clear_flux_maps": (C.c_int, [C.c_void_p]),
    "st_b200_flux_counts": (C.c_int, [C.c_void_p, C.c_int, _u64p]),
    "st_b200_run_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "st_b200_element_counts": (C.c_int, [C.c_void_p, C.c_int, _u64p, _u64p, _u64p]),
    "st_b200_flux_stats": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(FluxStats)]),
    "st_b200_set_save_stage_data": (C.c_int, [C.c_void_p, C.c_int]),
    "st_b200_stage_data_sizes": (C.c_int, [C.c_void_p, C.POINTER(st_uint_t), C.POINTER(st_uint_t)]),
    "st_b200_stage_data": (C.c_int, [C.c_void_p, c_double_p, c_double_p]),
    "st_b200_sim_run_replay": (C.c_int, [C.c_void_p, C.c_uint, st_uint_t, c_double_p, st_uint_t, c_double_p,
                                         C.c_void_p, C.c_void_p]),
    "st_b200_load_stinput": (C.c_int, [C.c_void_p, C.c_char_p]),
    "st_b200_set_max_sun_rays": (C.c_int, [C.c_void_p, C.c_ulonglong]),
    "st_b200_set_ranks": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "st_b200_sim_run_batch": (C.c_int, [C.c_void_p, C.c_uint, C.c_int, c_double_p, C.POINTER(st_uint_t), c_double_p]),
    "st_b200_batch_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Stats)]),
    "st_b200_batch_flux_counts": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _u64p]),
    "st_b200_batch_absorbed": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _u64p]),
    "st_b200_batch_sun_box": (C.c_int, [C.c_void_p, C.c_int, c_double_p, c_double_p, c_double_p, c_double_p]),
    "st_b200_write_rays": (C.c_int, [C.c_void_p, C.c_char_p]),
}


class B200Api(StApi):
    def stats(self, ctx) -> dict:
        s = Stats()
        self.st_b200_run_stats(ctx, C.byref(s))
        d = {k: getattr(s, k) for k, _ in Stats._fields_ if k != "stage_entries"}
        d["stage_entries"] = list(s.stage_entries)
        return d

    def flux(self, ctx, idx: int, nx: int, ny: int) -> np.ndarray:
        out = np.zeros(nx * ny, dtype=np.uint64)
        rc = self.st_b200_flux_counts(ctx, idx, out.ctypes.data_as(_u64p))
        if rc < 0:
            raise RuntimeError("st_b200_flux_counts failed")
        return out.reshape(ny, nx)

    def source_flux(self, ctx, idx: int, n_src: int, nx: int, ny: int) -> np.ndarray:
        """Counts of a per-source flux map: (n_src, ny, nx)."""
        out = np.zeros(n_src * nx * ny, dtype=np.uint64)
        if self.st_b200_flux_counts(ctx, idx, out.ctypes.data_as(_u64p)) < 0:
            raise RuntimeError("st_b200_flux_counts failed")
        return out.reshape(n_src, ny, nx)

    def flux_stats(self, ctx, idx: int, dni: float) -> dict:
        """Peak/min/mean flux, sigma, uniformity and uncertainties of flux map `idx`."""
        s = FluxStats()
        if self.st_b200_flux_stats(ctx, idx, dni, C.byref(s)) < 0:
            raise RuntimeError("st_b200_flux_stats failed: " + "; ".join(self.messages(ctx)))
        return {k: getattr(s, k) for k, _ in FluxStats._fields_}

    def stage_data(self, ctx):
        """(s0, s1) of the last run with stage-data saving on: arrays (n0, 8) and (n1, 7)."""
        n0, n1 = st_uint_t(), st_uint_t()
        self.st_b200_stage_data_sizes(ctx, C.byref(n0), C.byref(n1))
        s0 = np.zeros((n0.value, 8))
        s1 = np.zeros((n1.value, 7))
        self.st_b200_stage_data(ctx, s0.ctypes.data_as(c_double_p), s1.ctypes.data_as(c_double_p))
        return s0, s1

    def run_replay(self, ctx, seed: int, s0: np.ndarray, s1: np.ndarray) -> int:
        """Trace the stages after the first from saved stage data (st_b200_sim_run_replay)."""
        s0 = np.ascontiguousarray(s0, dtype=np.float64).reshape(-1, 8)
        s1 = np.ascontiguousarray(s1, dtype=np.float64).reshape(-1, 7)
        return self.st_b200_sim_run_replay(ctx, seed, len(s0), s0.ctypes.data_as(c_double_p), len(s1),
                                           s1.ctypes.data_as(c_double_p), None, None)

    def element_counts(self, ctx, stage: int, n: int):
        a = np.zeros(n, dtype=np.uint64)
        b = np.zeros(n, dtype=np.uint64)
        c = np.zeros(n, dtype=np.uint64)
        self.st_b200_element_counts(ctx, stage, a.ctypes.data_as(_u64p), b.ctypes.data_as(_u64p), c.ctypes.data_as(_u64p))
        return a, b, c

    def run_batch(self, ctx, seed: int, sun_xyz, hits, track_target=None) -> int:
        """st_b200_sim_run_batch: K sun positions (K x 3) with their hit counts; position k
        draws from the streams of seed + k."""
        sun = np.ascontiguousarray(sun_xyz, dtype=np.float64).reshape(-1, 3)
        h = np.ascontiguousarray(hits, dtype=np.uint64).reshape(-1)
        if len(h) != len(sun):
            raise ValueError("one hit count per sun position")
        tgt = None if track_target is None else np.ascontiguousarray(track_target, dtype=np.float64)
        return self.st_b200_sim_run_batch(ctx, seed, len(sun), sun.ctypes.data_as(c_double_p),
                                          h.ctypes.data_as(C.POINTER(st_uint_t)),
                                          None if tgt is None else tgt.ctypes.data_as(c_double_p))

    def batch_stats(self, ctx, position: int) -> dict:
        s = Stats()
        if self.st_b200_batch_stats(ctx, position, C.byref(s)) < 0:
            raise RuntimeError("st_b200_batch_stats failed")
        d = {k: getattr(s, k) for k, _ in Stats._fields_ if k != "stage_entries"}
        d["stage_entries"] = list(s.stage_entries)
        return d

    def batch_flux(self, ctx, idx: int, position: int, nx: int, ny: int) -> np.ndarray:
        out = np.zeros(nx * ny, dtype=np.uint64)
        if self.st_b200_batch_flux_counts(ctx, idx, position, out.ctypes.data_as(_u64p)) < 0:
            raise RuntimeError("st_b200_batch_flux_counts failed")
        return out.reshape(ny, nx)

    def batch_absorbed(self, ctx, position: int, stage: int, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.uint64)
        if self.st_b200_batch_absorbed(ctx, position, stage, out.ctypes.data_as(_u64p)) < 0:
            raise RuntimeError("st_b200_batch_absorbed failed")
        return out

    def batch_sun_box(self, ctx, position: int):
        v = [C.c_double() for _ in range(4)]
        if self.st_b200_batch_sun_box(ctx, position, *[C.byref(x) for x in v]) < 0:
            raise RuntimeError("st_b200_batch_sun_box failed")
        return tuple(x.value for x in v)

    def explicit_rays(self, ctx, pos: np.ndarray, cos: np.ndarray) -> int:
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        cos = np.ascontiguousarray(cos, dtype=np.float64)
        self._ex_keep = (pos, cos)
        return self.st_b200_explicit_rays(ctx, len(pos), pos.ctypes.data_as(c_double_p), cos.ctypes.data_as(c_double_p))


_API = None


def load(path: str | None = None) -> B200Api:
    """Bind the built library; raises FileNotFoundError when it is missing."""
    global _API
    p = path or LIB_PATH
    if path is None and _API is not None:
        return _API
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} is not built; run `python -m soltrace_b200.build`")
    api = B200Api(C.CDLL(p), EXTENSIONS)
    if path is None:
        _API = api
    return api
