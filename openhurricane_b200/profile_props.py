"""Mixture-property kernel timing on the 53-species mechanism, for
profiling with ncu.

    python -m openhurricane_b200.profile_props NCELLS

Seeded cells of the large workload (T U[800, 2800] K, p U[0.5, 10] atm,
Y ~ Dirichlet(0.3)); three untimed launches, then five launches timed with
CUDA events after a 256 MiB L2 flush each; prints one JSON line (median
time, cells/s, algorithmic GB/s).
"""
import json
import sys

import numpy as np
import torch

from . import workloads
from .chemistry import Mechanism


def main(argv):
    n = int(argv[0]) if argv else 262144
    _, _, t = workloads.mechanism_files("large")
    c = workloads.large_cells(n, 3003)
    m = Mechanism(t)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    T, p, Y = d(c.T), d(c.p), d(c.Y)
    flush = torch.empty((256 << 20) // 4, dtype=torch.float32, device="cuda")
    for _ in range(3):
        m.properties(T, p, Y)
    times = []
    st = torch.cuda.current_stream()
    for k in range(5):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        m.properties(T, p, Y)
        b.record(st)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms = float(np.median(times))
    nsp = t.nsp
    nbytes = n * 8.0 * ((2 + nsp) + (2 * nsp + 3))
    print(json.dumps({"cells": n, "species": nsp, "ms": ms, "cells_per_s": n / (ms * 1e-3),
                      "algorithmic_bytes": nbytes, "GB_per_s": nbytes / (ms * 1e-3) / 1e9}))


if __name__ == "__main__":
    main(sys.argv[1:])
