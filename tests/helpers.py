"""Shared helpers for the parity tests."""
from __future__ import annotations

import hashlib

import numpy as np

from soltrace_b200 import scenes


def run_scene(api, sc, seed, setup=None):
    """Push `sc` into a fresh context of `api`, run, and return (n, records, sun stats, messages)."""
    ctx = api.st_create_context()
    try:
        scenes.push(api, ctx, sc)
        if setup:
            setup(api, ctx)
        n = api.run(ctx, seed)
        rec = api.records(ctx) if n > 0 else api.records(ctx)
        ss = api.sun_stats(ctx)
        msg = api.messages(ctx)
        extra = setup.collect(api, ctx) if setup is not None and hasattr(setup, "collect") else None
    finally:
        api.st_free_context(ctx)
    return n, rec, ss, msg, extra


def records_digest(rec: dict) -> str:
    """sha256 over the raw record arrays in readback order (x y z cx cy cz element stage raynum)."""
    h = hashlib.sha256()
    for k in ("x", "y", "z", "cx", "cy", "cz"):
        h.update(np.ascontiguousarray(rec[k], dtype="<f8").tobytes())
    for k in ("element", "stage", "raynum"):
        h.update(np.ascontiguousarray(rec[k], dtype="<i4").tobytes())
    return h.hexdigest()


def assert_same_records(a: dict, b: dict, pos_tol: float, rel_tol: float = 0.0, dir_tol: float = None):
    """Integer fields identical; positions within pos_tol + rel_tol * (scene size), the scene
    size being the largest coordinate in the records (round-off grows with the length of the
    path a ray has travelled, not with its final coordinate); directions within dir_tol."""
    assert len(a["x"]) == len(b["x"]), (len(a["x"]), len(b["x"]))
    for k in ("element", "stage", "raynum"):
        assert np.array_equal(a[k], b[k]), k
    scale = max(float(np.max(np.abs(b[k]))) for k in ("x", "y", "z")) if len(b["x"]) else 0.0
    for k in ("x", "y", "z"):
        tol = pos_tol + rel_tol * scale
        d = np.abs(a[k] - b[k])
        assert np.all(d <= tol), (k, float(d.max()), tol)
    dtol = pos_tol if dir_tol is None else dir_tol
    for k in ("cx", "cy", "cz"):
        d = np.abs(a[k] - b[k])
        assert np.all(d <= dtol + rel_tol), (k, float(d.max()))


def c_declarations(text: str) -> dict:
    """name -> (return type, [parameter types]) of every st_* function declared in a C header,
    with comments, export macros and parameter names removed and array parameters written
    as the pointers they decay to (double x[8] -> double*, double m[3][3] -> double(*)[3])."""
    import re
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    text = text.replace("STCORE_API", " ")
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(st_\w+)\s*\(((?:[^()]|\([^()]*\))*)\)\s*;", text):
        ret = " ".join(m.group(1).split()).replace(" *", "*")
        params = []
        body = m.group(3).strip()
        if body and body != "void":
            depth, cur, parts = 0, "", []
            for ch in body:
                if ch == "(":
                    depth += 1
                elif ch == ")":
                    depth -= 1
                if ch == "," and depth == 0:
                    parts.append(cur)
                    cur = ""
                else:
                    cur += ch
            parts.append(cur)
            for p in parts:
                p = " ".join(p.split())
                if "(*" in p:
                    params.append("fnptr")
                    continue
                dims = re.findall(r"\[\s*\d*\s*\]", p)
                p = re.sub(r"\[\s*\d*\s*\]", "", p).strip()
                # drop the parameter name (the last identifier, unless the type is bare)
                toks = re.findall(r"[A-Za-z_]\w*|\*", p)
                if len(toks) > 1 and re.match(r"[A-Za-z_]", toks[-1]) and toks[-1] not in ("int", "double", "char",
                                                                                          "st_uint_t", "st_context_t"):
                    toks = toks[:-1]
                t = " ".join(toks).replace(" *", "*")
                if len(dims) == 1:
                    t += "*"
                elif len(dims) == 2:
                    t += "(*)" + dims[1].replace(" ", "")
                params.append(t)
        out[m.group(2)] = (ret, params)
    return out
