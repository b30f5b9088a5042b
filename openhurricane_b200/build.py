"""Build the CUDA library in-tree: openhurricane_b200/libhurchem_b200.so.

nvcc compiles the kernels for sm_100a only (B200); each kernel-size variant
is a separate translation unit so the variants compile in parallel. The CUDA
runtime is linked statically, so loading the library needs no CUDA install.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libhurchem_b200.so")
OBJDIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
# translation units: the C ABI plus one file per kernel variant
UNITS = ["capi.cu", "variant_10.cu", "variant_16.cu", "variant_32.cu", "variant_54.cu",
         "variant_64.cu", "variant_t1.cu", "props.cu", "probe.cu", "mlp.cu", "surrogate.cu"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _sources() -> List[str]:
    out = []
    for root, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(root, f))
    out.append(os.path.join(HERE, "..", "include", "hurchem_b200.h"))
    return out


def up_to_date() -> bool:
    if not os.path.isfile(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources() if os.path.exists(s))


def build_library(force: bool = False, verbose: bool = False, extra: List[str] = ()) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()

    def compile_one(u):
        obj = os.path.join(OBJDIR, u.replace(".cu", ".o"))
        cmd = [cc, *ARCH, *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, u), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {u}:\n{r.stderr[-4000:]}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(len(UNITS), os.cpu_count() or 4)) as ex:
        res = list(ex.map(compile_one, UNITS))
    objs = [o for o, _ in res]
    if verbose:
        for _, log in res:
            print(log)
    tmp = OUT + ".tmp"
    cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    import sys
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
