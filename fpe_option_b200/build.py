"""In-tree build of libfpe_engine.so for sm_100a (nvcc cross-compiles without a GPU)."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = [os.path.join(_HERE, "csrc", "engine.cu"), os.path.join(_HERE, "csrc", "mlp.cu")]
DEPS = [os.path.join(_HERE, "csrc", f) for f in os.listdir(os.path.join(_HERE, "csrc"))]
OUT = os.path.join(_HERE, "libfpe_engine.so")
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    inc_dir = os.path.join(os.path.dirname(_HERE), "include")
    incs = [os.path.join(inc_dir, f) for f in os.listdir(inc_dir)] if os.path.isdir(inc_dir) else []
    return any(os.path.getmtime(p) > t for p in DEPS + incs if os.path.exists(p))


def build_library(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        nvcc = os.environ.get("NVCC", "nvcc")
        cmd = [nvcc, *NVCC_FLAGS, "-o", OUT, *SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT
