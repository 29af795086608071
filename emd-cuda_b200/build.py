"""Build libemdb200.so in-tree with nvcc for sm_100a.

The sift translation unit is compiled with ``-fmad=false``: the FP64 results
must equal the reference algorithm's unfused multiply/add sequence bit for
bit (the CPU oracle restates it without FMA).  Other units use the default.

Usage: python emd-cuda_b200/build.py [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libemdb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *ARCH, f"-I{INCLUDE}"]
# (source, extra flags, object name)
UNITS = [
    ("emd_sift.cu", ["-fmad=false"], "emd_sift"),
    # the same kernels computing in float (namespace emdb::f32)
    ("emd_sift.cu", ["-fmad=false", "-DEMDB_F32=1"], "emd_sift_f32"),
    ("emd_sched.cu", [], "emd_sched"),
    ("emdb_api.cu", [], "emdb_api"),
    ("emdb_noalloc.cu", [], "emdb_noalloc"),
    ("emdb_pack.cu", [], "emdb_pack"),
]
HEADERS = ["emdb_internal.cuh", "emdb_sched.cuh"]


def _nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _newer(src: list[str], dst: str) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src if os.path.exists(s))


def build(force: bool = False, verbose: bool = False, defines: list[str] | None = None,
          out: str | None = None) -> str:
    """Compile the units and link the library.  `defines` (e.g.
    ["EMDB_LOAD_CLOCKS=1"]) and `out` build a variant library elsewhere,
    with its objects in a build folder of its own (the product build is
    unchanged)."""
    defines = list(defines or [])
    lib = out or LIB
    bdir = BUILD if not defines else os.path.join(BUILD, "_".join(d.replace("=", "") for d in defines))
    os.makedirs(bdir, exist_ok=True)
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "emdb200.h")]
    objs = []
    for src, extra, name in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, name + ".o")
        objs.append(o)
        if force or _newer([s, *hdrs, __file__], o):
            cmd = [nvcc, *COMMON, *extra, *[f"-D{d}" for d in defines], "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _newer(objs, lib):
        cmd = [nvcc, *ARCH, "-shared", "-o", lib, *objs, "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--define", action="append", default=[], help="extra -D for every unit")
    ap.add_argument("--out", default=None, help="library path (default: lib/libemdb200.so)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True, defines=a.define, out=a.out))
