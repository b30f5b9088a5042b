"""One integrator launch on seeded cells, for profiling with ncu.

    python -m openhurricane_b200.profile_case MECH NCELLS CAP KERNEL BLOCK [DT]

MECH is `small` (9 species / 21 reactions) or `large` (53 / 325); CAP caps
the Newton iterations of each cell (0: none) so that a capture stays short;
KERNEL / BLOCK as hc_set_tuning (0 automatic, 1 thread per cell, 2 cell
group, 3 mechanism-specialised thread per cell). Solver options atol 1e-11,
rtol 1e-4, dt 1e-6 s unless given.
"""
import ctypes as C
import sys

import numpy as np
import torch

from . import _capi, synth, workloads
from .chemistry import Mechanism


def main(argv):
    which, n, cap, kernel, block = argv[0], int(argv[1]), int(argv[2]), int(argv[3]), int(argv[4])
    dt = float(argv[5]) if len(argv) > 5 else 1e-6
    _, _, t = workloads.mechanism_files(which)
    c = workloads.small_cells(n, 1001) if which == "small" else workloads.large_cells(n, 3003)
    rho = synth.mixture_density(t.W, c)
    m = Mechanism(t)
    m.set_tuning(kernel, block)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    T, p, r, Y = d(c.T), d(c.p), d(rho), d(c.Y)
    dtt = torch.full((n,), dt, dtype=torch.float64, device="cuda")
    o = _capi.default_opts(max_newton_total=cap, **workloads.SOLVER_OPTS)
    vp = lambda x: C.c_void_p(x.data_ptr())
    sub = dtt.clone()
    cnt = _capi.HcCounters()
    rc = _capi.load().hc_integrate(m.handle, C.byref(o), n, vp(T), vp(p), vp(r), vp(Y), vp(dtt),
                                   1.0, vp(sub), None, None, C.addressof(cnt), None)
    _capi.check(rc, "hc_integrate")
    torch.cuda.synchronize()
    print("newton iterations", cnt.n_newton)


if __name__ == "__main__":
    main(sys.argv[1:])
