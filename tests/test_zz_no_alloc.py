"""hc_integrate_noalloc: the allocation-free variant of the compact
thread-per-cell integrator, against the allocating entry point on the same
kernel and inputs. Runs on a GPU; collected after every other test file."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

T_RTOL = 1e-6
Y_RTOL = 1e-5
Y_FLOOR = 1e-12


def _dev():
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch.device("cuda:0")


def _cells(tables, n, seed):
    from openhurricane_b200 import synth
    c = synth.dirichlet_cells(tables.nsp, n, seed=seed)
    return c.T, c.p, synth.mixture_density(tables.W, c), c.Y


def _run(entry, mech, opts, fields, n, dt):
    from openhurricane_b200 import _capi
    T0, p0, r0, Y0 = fields
    T, rho, Y = T0.clone(), r0.clone(), Y0.clone()
    sub = torch.full((n,), dt, dtype=torch.float64, device=T0.device)
    dtt = torch.full((n,), dt, dtype=torch.float64, device=T0.device)
    st = torch.zeros(n, dtype=torch.int32, device=T0.device)
    vp = lambda t: C.c_void_p(t.data_ptr())
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = _capi.load()
    if entry == "noalloc":
        rc = lib.hc_integrate_noalloc(mech.handle, C.byref(opts), n, vp(T), vp(p0), vp(rho), vp(Y),
                                      vp(dtt), 1.0, vp(sub), None, vp(st), s)
    else:
        rc = lib.hc_integrate(mech.handle, C.byref(opts), n, vp(T), vp(p0), vp(rho), vp(Y),
                              vp(dtt), 1.0, vp(sub), None, vp(st), None, s)
    _capi.check(rc, entry)
    torch.cuda.synchronize()
    return T.cpu().numpy(), rho.cpu().numpy(), Y.cpu().numpy(), sub.cpu().numpy(), st.cpu().numpy()


def _close(a, b):
    Ta, ra, Ya = a[0], a[1], a[2]
    Tb, rb, Yb = b[0], b[1], b[2]
    assert np.max(np.abs(Ta - Tb) / np.abs(Tb)) <= T_RTOL
    assert np.max(np.abs(ra - rb) / np.abs(rb)) <= T_RTOL
    assert np.max(np.abs(Ya - Yb) - Y_RTOL * np.abs(Yb) - Y_FLOOR) <= 0.0


def test_noalloc_matches_allocating_entry_point_twice_in_a_row(small):
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = small["tables"]
    mech = Mechanism(t)
    mech.set_tuning(4, 64)       # the allocating entry point on the same compact kernel
    n = 3000
    T, p, rho, Y = _cells(t, n, seed=515)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    fields = (d(T), d(p), d(rho), d(Y))
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)
    ref = _run("alloc", mech, opts, fields, n, 1e-6)
    # the first call may load the library's device image (which holds the
    # scratch array) under lazy module loading; the second must not change
    # the free device memory at all
    first = _run("noalloc", mech, opts, fields, n, 1e-6)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    second = _run("noalloc", mech, opts, fields, n, 1e-6)
    free1 = torch.cuda.mem_get_info()[0]
    _close(first, ref)
    _close(second, ref)
    assert np.array_equal(first[3], ref[3]) or np.allclose(first[3], ref[3], rtol=1e-6)
    assert np.array_equal(first[4], ref[4])
    assert free1 == free0, "device memory changed across the allocation-free calls"


def test_noalloc_rejects_more_cells_than_its_scratch(small):
    from openhurricane_b200 import _capi
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    mech = Mechanism(small["tables"])
    n = _capi.NOALLOC_MAX_CELLS + 1
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    Y = torch.zeros((small["tables"].nsp, n), dtype=torch.float64, device=dev)
    vp = lambda t: C.c_void_p(t.data_ptr())
    lib = _capi.load()
    rc = lib.hc_integrate_noalloc(mech.handle, C.byref(_capi.default_opts()), n, vp(x), vp(x),
                                  vp(x), vp(Y), vp(x), 1.0, vp(x), None, None, None)
    assert rc == -1
    assert b"HC_NOALLOC_MAX_CELLS" in lib.hc_last_error()


def test_noalloc_replays_from_a_cuda_graph(small):
    """One eager call (looks the scratch array up), then the same call
    captured in a CUDA graph and replayed on restored inputs: bit-identical
    to the eager result, with no change of free device memory on replay."""
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = small["tables"]
    mech = Mechanism(t)
    mech.set_tuning(4, 64)
    n = 2048
    T0, p0, r0, Y0 = (torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
                      for a in _cells(t, n, seed=616))
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)
    eager = _run("noalloc", mech, opts, (T0, p0, r0, Y0), n, 1e-6)
    T, rho, Y = T0.clone(), r0.clone(), Y0.clone()
    dtt = torch.full((n,), 1e-6, dtype=torch.float64, device=dev)
    sub = dtt.clone()
    st = torch.zeros(n, dtype=torch.int32, device=dev)
    vp = lambda x: C.c_void_p(x.data_ptr())
    lib = _capi.load()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            rc = lib.hc_integrate_noalloc(mech.handle, C.byref(opts), n, vp(T), vp(p0), vp(rho), vp(Y),
                                          vp(dtt), 1.0, vp(sub), None, vp(st),
                                          C.c_void_p(side.cuda_stream))
            assert rc == 0, lib.hc_last_error()
    torch.cuda.current_stream().wait_stream(side)
    # capture recorded the work without running it: restore and replay
    T.copy_(T0)
    rho.copy_(r0)
    Y.copy_(Y0)
    sub.fill_(1e-6)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    g.replay()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert np.array_equal(T.cpu().numpy(), eager[0])
    assert np.array_equal(rho.cpu().numpy(), eager[1])
    assert np.array_equal(Y.cpu().numpy(), eager[2])
    assert np.array_equal(st.cpu().numpy(), eager[4])
    assert free1 == free0
    del g
