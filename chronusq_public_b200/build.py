"""Build the in-tree CUDA engine ``libcqgpu.so`` for sm_100a.

    python -m chronusq_public_b200.build [--force]

Steps: generate the per-class ERI code (csrc/gen_eri.py -> csrc/_gen/eri_classes.cuh),
then compile csrc/engine.cu with nvcc into chronusq_public_b200/libcqgpu.so.  The build
is skipped when the library is newer than every source.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "_gen", "eri_classes.cuh")
OUT = os.path.join(HERE, "libcqgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
MAXL = 3

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-shared", "-Xcompiler", "-fPIC"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _sources():
    return (glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(CSRC, "*.py")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(OUT) or not os.path.exists(GEN):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, verbose: bool = True) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(os.path.dirname(GEN), exist_ok=True)
    subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_eri.py"), GEN, str(MAXL)])
    cmd = [_nvcc()] + NVCC_FLAGS + ["-o", OUT + ".tmp", os.path.join(CSRC, "engine.cu"),
                                    os.path.join(CSRC, "mlp.cu")]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
