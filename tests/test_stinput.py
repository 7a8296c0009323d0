"""The .stinput reader and .rays writer (st_b200_load_stinput, st_b200_write_rays) and the
strace_b200 command-line tracer.

Pin (CPU): scenes written as .stinput files are run by the reference's own CLI, strace
(coretrace/strace/main.cpp, built from its sources by `make -C oracle ref`), and by the
product's reader and writer on the CPU oracle in its reference-stream mode (which
reproduces the reference's records bit for bit).  The two .rays files must be identical
byte for byte: same scene read, same records, same text.

GPU: a scene read from its .stinput traces exactly as the same scene set through the C
API, and the CLI writes the same .rays as the library call.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from soltrace_b200 import scenes
from soltrace_b200.stinput import write_stinput

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRACE_REF = os.path.join(ROOT, "oracle", "_ref", "strace_ref")
CLI = os.path.join(ROOT, "soltrace_b200", "strace_b200")

CPU_CASES = ["dish", "trough", "sphere_circle", "hyperboloid", "parabola_hex", "parabola_irrtri", "torus",
             "cylinder", "spline", "sun_table", "sun_point", "optics_diffuse", "refl_table", "refraction",
             "virtual_stage", "tracethrough", "multi_element"]


def _scene(name, zoo_scenes):
    if name == "dish":
        return scenes.dish_scene(4000)
    if name == "trough":
        return scenes.trough_scene(3000)
    return zoo_scenes[name]


def _bind(lib):
    lib.lib.st_b200_load_stinput.restype = C.c_int
    lib.lib.st_b200_load_stinput.argtypes = [C.c_void_p, C.c_char_p]
    lib.lib.st_b200_write_rays.restype = C.c_int
    lib.lib.st_b200_write_rays.argtypes = [C.c_void_p, C.c_char_p]
    return lib.lib.st_b200_load_stinput, lib.lib.st_b200_write_rays


@pytest.mark.parametrize("name", CPU_CASES)
def test_rays_file_matches_reference_cli(oracle, zoo_scenes, tmp_path, name):
    if not os.path.exists(STRACE_REF):
        pytest.skip("reference CLI not built (make -C oracle ref)")
    sc = _scene(name, zoo_scenes)
    seed = 17
    path = write_stinput(sc, str(tmp_path / f"{name}.stinput"))
    args = [STRACE_REF, path, str(sc.raycount), str(sc.raymax), str(seed), str(int(sc.sunshape_errors)),
            str(int(sc.optical_errors)), "0"]
    subprocess.run(args, cwd=str(tmp_path), check=True, capture_output=True, timeout=600)
    want = open(path + ".rays", "rb").read()

    load, write = _bind(oracle)
    ctx = oracle.st_create_context()
    try:
        oracle.st_oracle_set_rng(ctx, 0)
        assert load(ctx, path.encode()) == 1, oracle.messages(ctx)
        oracle.st_sim_params(ctx, sc.raycount, sc.raymax, 0)
        oracle.st_sim_errors(ctx, int(sc.sunshape_errors), int(sc.optical_errors))
        assert oracle.run(ctx, seed) >= 0, oracle.messages(ctx)
        out = str(tmp_path / f"{name}.mine.rays")
        assert write(ctx, out.encode()) == 1
    finally:
        oracle.st_free_context(ctx)
    got = open(out, "rb").read()
    assert got == want


@pytest.mark.parametrize("text,why", [
    ("SUN\tPTSRC\t0\n", "must start with"),
    ("# SOLTRACE VERSION 3.1.0 INPUT FILE\nSUN\tPTSRC\t0\tSHAPE\tp\tSIGMA\t4\tHALFWIDTH\t4\n", "XYZ"),
    ("# SOLTRACE VERSION 3.1.0 INPUT FILE\nSUN\tPTSRC\t0\tSHAPE\tp\tSIGMA\t4\tHALFWIDTH\t4\n"
     "XYZ\t0\t0\t100\tUSELDH\t0\tLDH\t0\t0\t0\nUSER SHAPE DATA\t0\nOPTICS LIST COUNT\t0\nSTAGE LIST COUNT\t1\n"
     "STAGE\tXYZ\t0\t0\t0\tAIM\t0\t0\t1\tZROT\t0\tVIRTUAL\t0\tMULTIHIT\t1\tELEMENTS\t1\tTRACETHROUGH\t0\nname\n"
     "1\t0\t0\t0\n", "too few fields"),
])
def test_reader_rejects_malformed_files(oracle, tmp_path, text, why):
    p = tmp_path / "bad.stinput"
    p.write_text(text)
    load, _ = _bind(oracle)
    ctx = oracle.st_create_context()
    try:
        assert load(ctx, str(p).encode()) == -1
        assert any(why in m for m in oracle.messages(ctx)), oracle.messages(ctx)
    finally:
        oracle.st_free_context(ctx)


def _records(api, ctx):
    r = api.records(ctx)
    return {k: np.asarray(v) for k, v in r.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["dish", "trough", "torus", "spline", "refraction", "tracethrough"])
def test_loaded_scene_traces_like_pushed_scene(product, zoo_scenes, tmp_path, name):
    sc = _scene(name, zoo_scenes)
    path = write_stinput(sc, str(tmp_path / f"{name}.stinput"))
    load, write = _bind(product)
    res = []
    for how in ("push", "file"):
        ctx = product.st_create_context()
        try:
            if how == "push":
                scenes.push(product, ctx, sc)
            else:
                assert load(ctx, path.encode()) == 1, product.messages(ctx)
                product.st_sim_params(ctx, sc.raycount, sc.raymax, int(sc.dynamic_group))
                product.st_sim_errors(ctx, int(sc.sunshape_errors), int(sc.optical_errors))
            product.st_b200_set_precision(ctx, 0)
            assert product.run(ctx, 23) > 0, product.messages(ctx)
            res.append(_records(product, ctx))
            if how == "file":
                assert write(ctx, str(tmp_path / "lib.rays").encode()) == 1
        finally:
            product.st_free_context(ctx)
    for k in res[0]:
        np.testing.assert_array_equal(res[0][k], res[1][k], err_msg=k)
    # the CLI: same file, same seed -> the same .rays as the library call
    proc = subprocess.run([CLI, path, str(sc.raycount), str(sc.raymax), "23", str(int(sc.sunshape_errors)),
                           str(int(sc.optical_errors)), "0"], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr
    assert open(path + ".rays", "rb").read() == open(tmp_path / "lib.rays", "rb").read()
