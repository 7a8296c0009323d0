import ctypes as C
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

ORACLE_SO = os.path.join(ROOT, "oracle", "_ref", "st_oracle.so")
REFERENCE_SO = os.path.join(ROOT, "oracle", "_ref", "coretrace_ref.so")

ORACLE_EXTRA = {
    "st_oracle_set_rng": (C.c_int, [C.c_void_p, C.c_int]),
    "st_oracle_explicit_rays": (C.c_int, [C.c_void_p, C.c_ulong, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "st_oracle_flux": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_int, C.POINTER(C.c_ulonglong)]),
    "st_oracle_sun_rays": (C.c_ulong, [C.c_void_p]),
}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA product")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (test infrastructure).  Built from oracle/ if missing."""
    from soltrace_b200.capi import StApi
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    return StApi(ORACLE_SO, ORACLE_EXTRA)


@pytest.fixture(scope="session")
def reference():
    """The reference coretrace built from its own sources (oracle/Makefile `ref`), if present."""
    from soltrace_b200.capi import StApi
    if not os.path.exists(REFERENCE_SO):
        pytest.skip("reference library not built (make -C oracle ref)")
    return StApi(REFERENCE_SO)


@pytest.fixture(scope="session")
def product():
    from soltrace_b200.lib import load
    return load()


@pytest.fixture(scope="session")
def zoo_scenes(tmp_path_factory):
    from scene_zoo import zoo
    return zoo(str(tmp_path_factory.mktemp("zoo")))
