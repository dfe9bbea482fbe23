"""Build ``emerge_b200/libemgpu.so`` for sm_100a with nvcc (in-tree).

The element kernel is compiled once per (material kind, precision) from
``element_inst.cu`` so the six heavy instances build in parallel; everything
is linked into one shared library with a C ABI (``include/emgpu.h``).

    python -m emerge_b200.build [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libemgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "--diag-suppress", "177"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _units():
    units = [("api", "api.cu", []), ("plan", "plan.cu", []), ("gather", "gather.cu", []),
             ("noalloc", "noalloc.cu", []), ("robin", "robin.cu", []), ("extend", "extend.cu", []),
             ("select", "select.cu", []), ("postproc", "postproc.cu", ["-fmad=false"]),
             ("coo", "coo.cu", []), ("solve", "solve.cu", []),
             ("heat", "heat.cu", ["-fmad=false"])]
    for form in (0, 1, 2):
        for kind in (0, 1, 2):
            units.append((f"element_{form}_{kind}", "element_inst.cu", [f"-DEMG_FORM={form}", f"-DEMG_KIND={kind}"]))
    return units


def _sources_mtime() -> float:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    files.append(os.path.join(os.path.dirname(HERE), "include", "emgpu.h"))
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    """Compile (if stale) and return the path of libemgpu.so."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _sources_mtime():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    units = _units()

    def compile_unit(u):
        name, src, defs = u
        obj = os.path.join(BUILD, name + ".o")
        cmd = [nvcc, *ARCH, *FLAGS, *defs, "-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {name}:\n{r.stderr}")
        return obj, r.stderr

    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        results = list(ex.map(compile_unit, units))
    objs = [o for o, _ in results]
    with open(os.path.join(BUILD, "ptxas.log"), "w") as f:
        for (name, _, _), (_, log) in zip(units, results):
            f.write(f"==== {name}\n{log}\n")
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    args = ap.parse_args()
    build(force=args.force, jobs=args.jobs, verbose=True)
    sys.exit(0)
