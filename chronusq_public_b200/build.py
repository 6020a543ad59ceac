"""Build the in-tree CUDA engine ``libcqgpu.so`` for sm_100a.

    python -m chronusq_public_b200.build [--force]

Steps: generate the per-class ERI code (csrc/gen_eri.py -> csrc/_gen/eri_classes.cuh),
compile the translation units in parallel -- csrc/engine.cu (C ABI, screening, list build),
csrc/mlp.cu (learned-guess kernels), csrc/eri_part.cu once per share of the quartet
classes (-DCQG_PART=0..NPART-1) and csrc/eri_fused.cu (the class-fused kernel) -- and link them with nvcc into
chronusq_public_b200/libcqgpu.so.  The build is skipped when the library is newer than
every source.
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
              "-Xcompiler", "-fPIC"]
NPART = 8          # shares of the quartet-class kernels (CQG_NPART in csrc/engine_impl.cuh)


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _sources():
    return (glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(CSRC, "*.h")) +
            glob.glob(os.path.join(CSRC, "*.py")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(OUT) or not os.path.exists(GEN):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, verbose: bool = True, extra_flags=()) -> str:
    """Compile and link the engine; `extra_flags` are added to every nvcc compile (for
    example ``-Xptxas -v``), whose output is printed."""
    if not force and up_to_date():
        return OUT
    os.makedirs(os.path.dirname(GEN), exist_ok=True)
    subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_eri.py"), GEN, str(MAXL)])
    objdir = os.path.join(CSRC, "_gen", "obj")
    os.makedirs(objdir, exist_ok=True)
    units = [("engine", os.path.join(CSRC, "engine.cu"), []), ("mlp", os.path.join(CSRC, "mlp.cu"), [])]
    units += [("eri_part%d" % k, os.path.join(CSRC, "eri_part.cu"), ["-DCQG_PART=%d" % k]) for k in range(NPART)]
    units += [("eri_fused", os.path.join(CSRC, "eri_fused.cu"), [])]
    jobs = []
    for name, src, defs in units:
        obj = os.path.join(objdir, name + ".o")
        cmd = [_nvcc()] + NVCC_FLAGS + list(extra_flags) + defs + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append((obj, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for obj, cmd, proc in jobs:
        out, _ = proc.communicate()
        if out and (verbose or proc.returncode):
            print(out, end="", flush=True)
        if proc.returncode:
            failed.append(obj)
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc", output="failed: " + ", ".join(failed))
    link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
            "-o", OUT + ".tmp"] + [obj for obj, _, _ in jobs]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.check_call(link)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    flags = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else []
    build(force="--force" in sys.argv or bool(flags), extra_flags=flags)
