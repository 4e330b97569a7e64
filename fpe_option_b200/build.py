"""In-tree build of libfpe_engine.so for sm_100a (nvcc cross-compiles without a GPU).

Every translation unit compiles to its own object in parallel (the two Radau
kernel instantiations are the slowest), then one link step makes the library.
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

_HERE = os.path.dirname(os.path.abspath(__file__))
_CSRC = os.path.join(_HERE, "csrc")
SOURCES = [os.path.join(_CSRC, f) for f in ("engine.cu", "radau_f32.cu", "radau_f64.cu", "mlp.cu")]
DEPS = [os.path.join(_CSRC, f) for f in os.listdir(_CSRC)]
OUT = os.path.join(_HERE, "libfpe_engine.so")
OBJ_DIR = os.path.join(_HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", *ARCH, "-Xcompiler", "-fPIC"]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    inc_dir = os.path.join(os.path.dirname(_HERE), "include")
    incs = [os.path.join(inc_dir, f) for f in os.listdir(inc_dir)] if os.path.isdir(inc_dir) else []
    return any(os.path.getmtime(p) > t for p in DEPS + incs + [__file__] if os.path.exists(p))


def build_library(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        nvcc = os.environ.get("NVCC", "nvcc")
        os.makedirs(OBJ_DIR, exist_ok=True)
        objs = [os.path.join(OBJ_DIR, os.path.basename(s)[:-3] + ".o") for s in SOURCES]
        cmds = [[nvcc, *NVCC_FLAGS, "-c", "-o", o, s] for s, o in zip(SOURCES, objs)]
        if verbose:
            for c in cmds:
                print(" ".join(c))
        with ThreadPoolExecutor(len(cmds)) as ex:
            for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
                if r.returncode != 0:
                    raise RuntimeError(f"nvcc failed:\n{r.stderr[-4000:]}")
        link = [nvcc, *ARCH, "-shared", "-o", OUT, *objs]
        subprocess.run(link, check=True)
    return OUT
