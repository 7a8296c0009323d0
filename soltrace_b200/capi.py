"""ctypes binding of the SolTrace flat C API (coretrace/stapi.h:68-176).

`StApi` wraps any shared library that exports that API: the CUDA product
(`coretrace_api.so` built from soltrace_b200/csrc), or another implementation of
the same ABI.  Argument types follow the header exactly (st_uint_t is
`unsigned long`, characters are passed as C `char`).
"""
from __future__ import annotations

import ctypes as C
import numpy as np

st_uint_t = C.c_ulong
c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)

# int (*)(st_uint_t ntracedtotal, st_uint_t ntraced, st_uint_t ntotrace,
#         st_uint_t curstage, st_uint_t nstages, void *data)
PROGRESS_CB = C.CFUNCTYPE(C.c_int, st_uint_t, st_uint_t, st_uint_t, st_uint_t, st_uint_t, C.c_void_p)

_SIGNATURES = {
    "st_create_context": (C.c_void_p, []),
    "st_free_context": (C.c_int, [C.c_void_p]),
    "st_num_messages": (C.c_int, [C.c_void_p]),
    "st_message": (C.c_char_p, [C.c_void_p, st_uint_t]),
    "st_clear_messages": (None, [C.c_void_p]),
    "st_num_optics": (C.c_int, [C.c_void_p]),
    "st_add_optic": (C.c_int, [C.c_void_p, C.c_char_p]),
    "st_delete_optic": (C.c_int, [C.c_void_p, st_uint_t]),
    "st_clear_optics": (C.c_int, [C.c_void_p]),
    "st_optic": (C.c_int, [C.c_void_p, st_uint_t, C.c_int, C.c_char, C.c_int, C.c_int, C.c_int,
                           C.c_double, C.c_double, C.c_double, C.c_double, c_double_p,
                           C.c_double, C.c_double, C.c_int, C.c_int, c_double_p, c_double_p,
                           C.c_int, C.c_int, c_double_p, c_double_p]),
    "st_num_stages": (C.c_int, [C.c_void_p]),
    "st_add_stage": (C.c_int, [C.c_void_p]),
    "st_add_stages": (C.c_int, [C.c_void_p, st_uint_t]),
    "st_delete_stage": (C.c_int, [C.c_void_p, st_uint_t]),
    "st_clear_stages": (C.c_int, [C.c_void_p]),
    "st_stage_xyz": (C.c_int, [C.c_void_p, st_uint_t, C.c_double, C.c_double, C.c_double]),
    "st_stage_aim": (C.c_int, [C.c_void_p, st_uint_t, C.c_double, C.c_double, C.c_double]),
    "st_stage_zrot": (C.c_int, [C.c_void_p, st_uint_t, C.c_double]),
    "st_stage_flags": (C.c_int, [C.c_void_p, st_uint_t, C.c_int, C.c_int, C.c_int]),
    "st_num_elements": (C.c_int, [C.c_void_p, st_uint_t]),
    "st_add_element": (C.c_int, [C.c_void_p, st_uint_t]),
    "st_add_elements": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t]),
    "st_delete_element": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t]),
    "st_clear_elements": (C.c_int, [C.c_void_p, st_uint_t]),
    "st_element_enabled": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_int]),
    "st_element_xyz": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_double, C.c_double, C.c_double]),
    "st_element_aim": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_double, C.c_double, C.c_double]),
    "st_element_zrot": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_double]),
    "st_element_aperture": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_char]),
    "st_element_aperture_params": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, c_double_p]),
    "st_element_surface": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_char]),
    "st_element_surface_params": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, c_double_p]),
    "st_element_surface_file": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_char_p]),
    "st_element_interaction": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_int]),
    "st_element_optic": (C.c_int, [C.c_void_p, st_uint_t, st_uint_t, C.c_char_p]),
    "st_sun": (C.c_int, [C.c_void_p, C.c_int, C.c_char, C.c_double]),
    "st_sun_xyz": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "st_sun_position": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                  c_double_p, c_double_p, c_double_p]),
    "st_sun_userdata": (C.c_int, [C.c_void_p, st_uint_t, c_double_p, c_double_p]),
    "st_num_intersections": (C.c_int, [C.c_void_p]),
    "st_locations": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p]),
    "st_cosines": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p]),
    "st_elementmap": (C.c_int, [C.c_void_p, c_int_p]),
    "st_stagemap": (C.c_int, [C.c_void_p, c_int_p]),
    "st_raynumbers": (C.c_int, [C.c_void_p, c_int_p]),
    "st_sun_stats": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, c_double_p, c_int_p]),
    "st_sim_params": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "st_sim_errors": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "st_sim_run": (C.c_int, [C.c_void_p, C.c_uint, PROGRESS_CB, C.c_void_p]),
    "st_calc_euler_angles": (None, [c_double_p, c_double_p, C.c_double, c_double_p]),
    "st_transform_to_local": (None, [c_double_p] * 6),
    "st_transform_to_reference": (None, [c_double_p] * 6),
    "st_matrix_vector_mult": (None, [c_double_p] * 3),
    "st_calc_transform_matrices": (None, [c_double_p] * 3),
    "st_matrix_transpose": (None, [c_double_p] * 2),
}

#: every entry point of the reference header, in header order
STAPI_FUNCTIONS = tuple(_SIGNATURES)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(c_double_p)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(c_int_p)


class StApi:
    """Typed view of one library exporting the stapi.h functions."""

    def __init__(self, lib: C.CDLL | str, extra: dict | None = None):
        self.lib = C.CDLL(lib) if isinstance(lib, str) else lib
        sigs = dict(_SIGNATURES)
        if extra:
            sigs.update(extra)
        for name, (res, args) in sigs.items():
            fn = getattr(self.lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)

    def has(self, name: str) -> bool:
        return hasattr(self, name)

    # ---- readback helpers ----
    def messages(self, ctx) -> list[str]:
        n = self.st_num_messages(ctx)
        return [self.st_message(ctx, i).decode(errors="replace") for i in range(max(n, 0))]

    def records(self, ctx) -> dict:
        n = self.st_num_intersections(ctx)
        out = {k: np.zeros(max(n, 0)) for k in ("x", "y", "z", "cx", "cy", "cz")}
        for k in ("element", "stage", "raynum"):
            out[k] = np.zeros(max(n, 0), dtype=np.int32)
        if n > 0:
            self.st_locations(ctx, dptr(out["x"]), dptr(out["y"]), dptr(out["z"]))
            self.st_cosines(ctx, dptr(out["cx"]), dptr(out["cy"]), dptr(out["cz"]))
            self.st_elementmap(ctx, iptr(out["element"]))
            self.st_stagemap(ctx, iptr(out["stage"]))
            self.st_raynumbers(ctx, iptr(out["raynum"]))
        return out

    def sun_stats(self, ctx) -> dict:
        v = [C.c_double() for _ in range(4)]
        n = C.c_int()
        self.st_sun_stats(ctx, *[C.byref(x) for x in v], C.byref(n))
        return {"xmin": v[0].value, "xmax": v[1].value, "ymin": v[2].value, "ymax": v[3].value,
                "nsunrays": n.value}

    def run(self, ctx, seed: int, callback=None) -> int:
        # no callback -> NULL function pointer (the trace then never calls back)
        cb = PROGRESS_CB(callback) if callback else PROGRESS_CB()
        self._last_cb = cb  # keep alive for the duration of the call
        return self.st_sim_run(ctx, seed, cb, None)
