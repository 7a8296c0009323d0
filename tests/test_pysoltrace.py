"""The reference's Python front end (app/deploy/api/pysoltrace.py), unmodified, on the
product library: the drop-in as its main caller uses it.

pysoltrace loads coretrace_api.so from its working directory (pysoltrace.py:1518-1531); here
the working directory holds a link to soltrace_b200/coretrace_api.so.  The front end and the
tower demo are copied from the reference checkout by the oracle recipe (`make -C oracle ref`,
into oracle/_ref/pysoltrace); without them these tests skip.  Each case runs in a fresh Python
process (tests/pysoltrace_driver.py): pysoltrace's multi-thread mode forks worker processes,
which must not inherit a CUDA context.

* dish: a parabolic dish and flat receiver built through pysoltrace's objects, one thread,
  seed 123.  Its ray table (PT.raydata) equals, record for record, the oracle's trace (per-ray
  streams) of the system pysoltrace's own write_soltrace_input_file wrote: element, stage and
  ray number equal, positions within 1e-9 m.  The flux map pysoltrace computes from that table
  (plot_flux, pysoltrace.py:1916-1960) equals the oracle's kind-0 bins of its records, up to
  hits within rounding of a bin edge.
* tower: the reference's tower demo script as shipped (1e6 hits over 8 worker processes):
  it completes, the workers' tables hold the 1e6 first-stage hits, merged with ray numbers
  offset per worker (pysoltrace.py:1636-1645), and its 50 x 50 flux map holds every absorbed
  hit.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import assert_same_records

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PYS = os.path.join(ROOT, "oracle", "_ref", "pysoltrace")
DRIVER = os.path.join(ROOT, "tests", "pysoltrace_driver.py")
LIB = os.path.join(ROOT, "soltrace_b200", "coretrace_api.so")


def _drive(tmp_path, case, timeout=600):
    if not os.path.exists(os.path.join(PYS, "pysoltrace.py")):
        pytest.skip("pysoltrace not copied (make -C oracle ref)")
    os.symlink(LIB, tmp_path / "coretrace_api.so")
    out = tmp_path / "out.npz"
    proc = subprocess.run([sys.executable, DRIVER, case, str(tmp_path), PYS, str(out)], capture_output=True,
                          text=True, timeout=timeout)
    assert proc.returncode == 0, proc.stdout[-3000:] + proc.stderr[-3000:]
    return dict(np.load(out))


def test_pysoltrace_dish_equals_oracle(tmp_path, oracle):
    got = _drive(tmp_path, "dish")
    assert int(got["res"]) > 0
    # the oracle traces the system pysoltrace wrote, read back by the .stinput front end
    load = oracle.lib.st_b200_load_stinput
    load.restype, load.argtypes = C.c_int, [C.c_void_p, C.c_char_p]
    cwd = os.getcwd()
    os.chdir(tmp_path)
    ctx = oracle.st_create_context()
    try:
        assert load(ctx, b"dish.stinput") == 1, oracle.messages(ctx)
        oracle.st_oracle_set_rng(ctx, 1)
        oracle.st_sim_params(ctx, 20000, 2_000_000, 0)
        oracle.st_sim_errors(ctx, 1, 1)
        assert oracle.run(ctx, 123) > 0
        want = oracle.records(ctx)
        sun = oracle.sun_stats(ctx)
        bins = np.zeros(25 * 25, dtype=np.uint64)
        oracle.st_oracle_flux(ctx, 2, 1, 0, 25, 25, -0.25, 0.25, -0.25, 0.25, 1,
                              bins.ctypes.data_as(C.POINTER(C.c_ulonglong)))
    finally:
        oracle.st_free_context(ctx)
        os.chdir(cwd)
    rec = {"x": got["loc"][:, 0], "y": got["loc"][:, 1], "z": got["loc"][:, 2], "cx": got["cos"][:, 0],
           "cy": got["cos"][:, 1], "cz": got["cos"][:, 2], "element": got["element"], "stage": got["stage"],
           "raynum": got["number"]}
    assert_same_records(rec, want, pos_tol=1e-9, rel_tol=2e-12, dir_tol=1e-9)
    assert got["sun"][4] == sun["nsunrays"]
    np.testing.assert_allclose(got["sun"][:4], [sun["xmin"], sun["xmax"], sun["ymin"], sun["ymax"]], rtol=1e-12)
    # pysoltrace's map, flux_st[ix, iy] += ppr / node area (its (ny, nx) array indexed [x, y])
    anode = (0.5 / 25) * (0.5 / 25)
    counts = np.rint(got["flux"] / (got["ppr"] / anode)).astype(np.int64)
    oracle_counts = bins.reshape(25, 25).T.astype(np.int64)  # [iy][ix] -> [ix][iy]
    assert counts.sum() == oracle_counts.sum() > 0
    assert np.abs(counts - oracle_counts).sum() <= 4


def test_pysoltrace_tower_demo_runs_as_shipped(tmp_path):
    got = _drive(tmp_path, "tower", timeout=900)
    assert (tmp_path / "simpletest.stinput").exists()
    # 1e6 first-stage hits split over the workers (125,000 each), numbered from 1 upwards
    assert int(np.sum(got["stage"] == 1)) == 1_000_000
    assert got["number"].min() == 1 and got["number"].max() >= 1_000_000 * 0.99
    absorbed = int(np.sum((got["stage"] == 2) & (got["element"] == -1)))
    flux = got["flux"]
    assert flux.shape == (50, 50) and absorbed > 0
    anode = (2.0 / 50) * (2.0 / 50)
    assert int(np.rint(flux.sum() / (got["ppr"] / anode))) == absorbed
