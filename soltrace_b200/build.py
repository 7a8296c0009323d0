"""Build coretrace_api.so (CUDA sm_100a + C++17) and the strace_b200 CLI in-tree.

    python -m soltrace_b200.build          # or: from soltrace_b200.build import build; build()

Every translation unit is compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`;
the FP64 kernels are compiled with -fmad=false so that double arithmetic rounds like
the reference's x86-64 build.  The CUDA runtime is linked statically, so the
library only needs the driver (libcuda) at load time.  Objects go to
soltrace_b200/_build/, the library to soltrace_b200/coretrace_api.so.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "coretrace_api.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=default",
          f"-I{INCLUDE}", f"-I{CSRC}", "--expt-relaxed-constexpr"]
UNITS = {
    "st_host.cpp": ["-x", "cu"],
    "st_run.cu": [],
    "st_kernels_fp64.cu": ["-fmad=false"],
    "st_kernels_mixed.cu": [],
    "st_kernels_common.cu": [],
    "st_noalloc.cu": [],
    "st_mlp.cu": [],
    "st_stinput.cpp": [],
}
CLI = os.path.join(HERE, "strace_b200")  # command-line tracer (csrc/strace_main.cpp)
HEADERS = ["st_scene.h", "st_device.cuh", "st_trace_impl.cuh", "st_host.h", "st_launch.h"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _digest(paths) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "stapi.h"), os.path.join(INCLUDE, "st_b200.h")]
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OUT, unit.rsplit(".", 1)[0] + ".o")
        stamp = obj + ".sha"
        dig = _digest([src] + hdrs) + " ".join(extra)
        if not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == dig:
            objs.append(obj)
            continue
        cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        with open(stamp, "w") as f:
            f.write(dig)
        objs.append(obj)
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    # the CLI links the library from its own directory
    cli_src = os.path.join(CSRC, "strace_main.cpp")
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", f"-I{INCLUDE}", cli_src, "-o", CLI, LIB,
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
