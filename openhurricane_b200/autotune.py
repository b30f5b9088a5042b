"""Autotuner for the integrator's launch shape.

Candidates are (kernel, block) pairs accepted by hc_set_tuning:
kernel 6 = warp per cell, kernel 7 = segment per cell (nsp + 1 <= 16;
256-thread blocks, the block argument is unused),
kernel 1 = thread per cell (nsp + 1 <= 16; block 32/64/128 threads),
kernel 3 = thread per cell generated for the mechanism (same limits),
kernel 4 = compact thread per cell (mechanism in the constant bank),
kernel 2 = cell group (32 lanes per cell up to 32 unknowns, 64 above; the
block argument is ignored).
Each candidate integrates the same sample of cells (a strided subset of the
caller's cells, restored before every trial) once untimed and `repeats`
times timed with CUDA events on the current stream; the fastest median wins
and is applied to the mechanism. Results are cached per (GPU name, nsp, nrc,
sample size) in memory and, when `cache_path` is given, in a JSON file.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import statistics
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _capi

_MEMO: Dict[str, dict] = {}


def candidates(nsp: int) -> List[Tuple[int, int]]:
    c = []
    if nsp + 1 <= 16:
        # warp and segment per cell (256-thread blocks: block unused), then
        # the thread-per-cell kernels
        c += [(6, 64), (7, 64), (4, 64), (4, 128), (3, 64), (1, 64)]
    c += [(2, 64)]      # the cell group's width is fixed by the variant; block is unused
    return c


def _key(mech, n: int) -> str:
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return f"{name}|{mech.nsp}|{mech.nrc}|{n}"


def autotune(mech, T: torch.Tensor, p: torch.Tensor, rho: torch.Tensor, Y: torch.Tensor,
             dt: torch.Tensor, opts=None, sample: int = 65536, repeats: int = 2,
             cands: Optional[Sequence[Tuple[int, int]]] = None,
             cache_path: Optional[str] = None) -> dict:
    """Pick and apply the fastest launch shape for these cells."""
    n = int(T.shape[0])
    stride = max(1, n // max(1, sample))
    idx = torch.arange(0, n, stride, device=T.device)[:sample]
    m = int(idx.shape[0])
    key = _key(mech, m)
    cache = {}
    if cache_path and os.path.isfile(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
    hit = _MEMO.get(key) or cache.get(key)
    if hit is not None:
        mech.set_tuning(hit["kernel"], hit["block"])
        return hit
    o = opts if opts is not None else _capi.default_opts()
    T0, p0, r0 = T[idx].contiguous(), p[idx].contiguous(), rho[idx].contiguous()
    Y0, d0 = Y[:, idx].contiguous(), dt[idx].contiguous()
    Tw, rw, Yw, sw = T0.clone(), r0.clone(), Y0.clone(), d0.clone()
    lib = _capi.load()
    stream = torch.cuda.current_stream()
    vp = lambda t: C.c_void_p(t.data_ptr())

    def run():
        Tw.copy_(T0)
        rw.copy_(r0)
        Yw.copy_(Y0)
        sw.copy_(d0)
        rc = lib.hc_integrate(mech.handle, C.byref(o), m, vp(Tw), vp(p0), vp(rw), vp(Yw),
                              vp(d0), 1.0, vp(sw), None, None, None,
                              C.c_void_p(stream.cuda_stream))
        _capi.check(rc, "hc_integrate")

    results = []
    for kernel, block in (cands or candidates(mech.nsp)):
        try:
            mech.set_tuning(kernel, block)
            run()
        except _capi.HcError:
            continue
        times = []
        for _ in range(repeats):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run()
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        results.append({"kernel": kernel, "block": block, "ms": statistics.median(times)})
    if not results:
        raise _capi.HcError("no launch shape ran for this mechanism")
    best = min(results, key=lambda r: r["ms"])
    out = {"kernel": best["kernel"], "block": best["block"], "ms": best["ms"],
           "sample_cells": m, "trials": results}
    mech.set_tuning(best["kernel"], best["block"])
    _MEMO[key] = out
    if cache_path:
        cache[key] = out
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, cache_path)
    return out
