"""In-tree build of libpbdose_b200.so for sm_100a (nvcc, no CMake).

    python -c "import importlib; importlib.import_module('gpu-proton-dose-engine_b200.build').build()"

Objects go to ``_build/`` inside the package; the shared library lands next to this
file so that it travels with the source tree.  The LUT builder is compiled with
``-fmad=false`` (its FP64 arithmetic rounds each product like the reference's NumPy);
the dose kernels keep FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpbdose_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I", INCLUDE]
SOURCES = {
    "api.cu": [],
    "lut.cu": ["-fmad=false"],
    "fwd_simt.cu": [],
    "fwd_f64.cu": [],
    "adj_simt.cu": [],
    "tc_fwd.cu": [],
    "tc_fwd16.cu": [],
    "noalloc.cu": [],
    "adj_tc.cu": [],
    "optim.cu": [],
    "gamma.cu": [],
}


def nvcc_path() -> str:
    p = shutil.which("nvcc")
    if p:
        return p
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=()) -> str:
    nvcc = nvcc_path()
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "pbdose_b200.h"))
    objs = []
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *ARCH, *COMMON, *flags, *extra_flags, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def ptxas_report(src: str = "fwd_simt.cu") -> str:
    """Register / spill / shared-memory report of one source (``-Xptxas -v``)."""
    nvcc = nvcc_path()
    flags = SOURCES.get(src, [])
    cmd = [nvcc, *ARCH, *COMMON, *flags, "-Xptxas", "-v", "-c", os.path.join(CSRC, src), "-o",
           os.devnull]
    r = subprocess.run(cmd, check=True, capture_output=True, text=True)
    return r.stderr


if __name__ == "__main__":
    print(build(verbose=True))
