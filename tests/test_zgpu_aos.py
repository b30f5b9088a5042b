"""Record-per-cell entry points (the reference's CUDA-path buffers) against
the species-major entry points on the same cells: the records are packed and
unpacked here in numpy exactly as the reference's callers do
(CUDAChemistrySource.cpp:73-81 and :377-399, laminarSpeciesSolverCUDA.cpp:326-330),
and the results must agree bit for bit, since the same kernels run on the
same numbers."""
import ctypes as C
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RU = (1.380649e-23 * 6.02214076e23) * 1e3


def _dev():
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch.device("cuda:0")


def _cells(tables, n, seed):
    from openhurricane_b200 import synth
    c = synth.dirichlet_cells(tables.nsp, n, seed=seed)
    return c.T, c.p, synth.mixture_density(tables.W, c), c.Y


def _ideal_gas_p(W, T, rho, Y):
    """rho Ru T sum_i Y_i / W_i, summed in species order like the kernel."""
    s = np.zeros_like(T)
    for i in range(Y.shape[0]):
        s = s + Y[i] / W[i]
    return rho * RU * T * s


def _pack_integration(T, Y, rho):
    """[T, Y_0..Y_{nsp-1}, rho] per cell (CUDAChemistrySource.cpp:377-385)."""
    return np.ascontiguousarray(np.concatenate([T[:, None], Y.T, rho[:, None]], axis=1))


def _pack_source(T, Y, rho):
    """[Y_0..Y_{nsp-1}, rho, T] per cell (CUDAChemistrySource.cpp:73-81)."""
    return np.ascontiguousarray(np.concatenate([Y.T, rho[:, None], T[:, None]], axis=1))


def _soa_integrate(mech, opts, T, p, rho, Y, dt, sub):
    from openhurricane_b200 import _capi
    dev = _dev()
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    Td, pd, rd, Yd, dtd, sd = d(T), d(p), d(rho), d(Y), d(dt), d(sub)
    n = T.shape[0]
    vp = lambda t: C.c_void_p(t.data_ptr())
    rc = _capi.load().hc_integrate(mech.handle, C.byref(opts), n, vp(Td), vp(pd), vp(rd), vp(Yd),
                                   vp(dtd), 1.0, vp(sd), None, None, None,
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _capi.check(rc, "hc_integrate")
    torch.cuda.synchronize()
    return Td.cpu().numpy(), rd.cpu().numpy(), Yd.cpu().numpy(), sd.cpu().numpy()


@pytest.mark.parametrize("return_ci", [1, 0])
@pytest.mark.parametrize("given_p", [True, False])
def test_integrate_records_match_species_major_fields(small, return_ci, given_p):
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = small["tables"]
    m = Mechanism(t)
    n = 301                           # not a multiple of the 32-cell tile
    T, p, rho, Y = _cells(t, n, seed=811)
    if not given_p:
        p = _ideal_gas_p(t.W, T, rho, Y)
    dt = np.full(n, 1e-7)
    sub = np.full(n, 1e-7)
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)
    Ts, rs, Ys, ss = _soa_integrate(m, opts, T, p, rho, Y, dt, sub)

    rec = torch.tensor(_pack_integration(T, Y, rho), device=dev)
    subd = torch.tensor(sub, device=dev)
    pd = torch.tensor(p, device=dev) if given_p else None
    st = m.integrate_aos(rec, torch.tensor(dt, device=dev), subd, p=pd, return_ci=bool(return_ci),
                         opts=opts)
    torch.cuda.synchronize()
    r = rec.cpu().numpy()
    assert np.array_equal(r[:, 0], Ts)
    assert np.array_equal(subd.cpu().numpy(), ss)
    assert not (st.cpu().numpy() & 0xC).any()        # HC_CELL_UNDERFLOW | HC_CELL_ITER_LIMIT
    if return_ci:
        c = (Ys * rs[None, :]) / t.W[:, None]
        assert np.array_equal(r[:, 1:-1], c.T)
        assert np.array_equal(r[:, -1], rho)          # the record's own rho is kept
    else:
        assert np.array_equal(r[:, 1:-1], Ys.T)
        assert np.array_equal(r[:, -1], rs)


def test_integrate_records_host_form_matches_device_form(small):
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = small["tables"]
    m = Mechanism(t)
    n = 77
    T, p, rho, Y = _cells(t, n, seed=812)
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)
    rec0 = _pack_integration(T, Y, rho)
    dt = np.full(n, 1e-7)
    rec_d = torch.tensor(rec0, device=dev)
    sub_d = torch.full((n,), 1e-7, dtype=torch.float64, device=dev)
    m.integrate_aos(rec_d, torch.tensor(dt, device=dev), sub_d, return_ci=True, opts=opts)
    torch.cuda.synchronize()
    rec_h = rec0.copy()
    sub_h = np.full(n, 1e-7)
    st_h = np.zeros(n, np.int32)
    rc = _capi.load().hc_integrate_aos_host(m.handle, C.byref(opts), n,
                                            rec_h.ctypes.data_as(C.c_void_p), None,
                                            dt.ctypes.data_as(C.c_void_p),
                                            sub_h.ctypes.data_as(C.c_void_p), 1,
                                            st_h.ctypes.data_as(C.c_void_p), None)
    assert rc == 0
    assert np.array_equal(rec_h, rec_d.cpu().numpy())
    assert np.array_equal(sub_h, sub_d.cpu().numpy())


def test_source_term_records_match_species_major_fields(large):
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = large["tables"]
    m = Mechanism(t)
    n = 4099
    T, p, rho, Y = _cells(t, n, seed=813)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    Ri = m.source_terms(d(T), d(p), d(rho), d(Y)).cpu().numpy()
    RRi = m.source_terms_aos(d(_pack_source(T, Y, rho)), p=d(p)).cpu().numpy()
    assert RRi.shape == (n, t.nsp)
    assert np.array_equal(RRi, Ri.T)
    pg = _ideal_gas_p(t.W, T, rho, Y)
    Ri_g = m.source_terms(d(T), d(pg), d(rho), d(Y)).cpu().numpy()
    assert np.array_equal(m.source_terms_aos(d(_pack_source(T, Y, rho))).cpu().numpy(), Ri_g.T)


def test_async_source_terms_return_before_the_results_and_overlap_host_work(small):
    """The host-buffer form only enqueues: the call returns while the copies
    and kernels are still running, host work proceeds, and after the stream
    is synchronised RRi holds the same numbers as the device form."""
    from openhurricane_b200 import _capi
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = small["tables"]
    m = Mechanism(t)
    n = 1 << 21
    rng = np.random.default_rng(814)
    Y = rng.dirichlet(np.ones(t.nsp), size=n).T.copy()
    T = rng.uniform(1000.0, 2500.0, n)
    rho = rng.uniform(0.1, 2.0, n)
    recs = torch.from_numpy(_pack_source(T, Y, rho)).pin_memory()
    RRi = torch.empty((n, t.nsp), dtype=torch.float64).pin_memory()
    ref = m.source_terms_aos(recs.to(dev)).cpu()
    s = torch.cuda.Stream()
    lib = _capi.load()
    # warm the workspace for this size (its first growth synchronises)
    assert lib.hc_source_terms_aos_async(m.handle, n, C.c_void_p(recs.data_ptr()), None,
                                         C.c_void_p(RRi.data_ptr()), C.c_void_p(s.cuda_stream)) == 0
    s.synchronize()
    RRi.zero_()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(s)
    t0 = time.perf_counter()
    rc = lib.hc_source_terms_aos_async(m.handle, n, C.c_void_p(recs.data_ptr()), None,
                                       C.c_void_p(RRi.data_ptr()), C.c_void_p(s.cuda_stream))
    t_call = time.perf_counter() - t0
    b.record(s)
    assert rc == 0
    host_work = float(np.sum(np.sqrt(np.arange(1 << 20, dtype=np.float64))))   # meanwhile
    s.synchronize()
    t_dev = a.elapsed_time(b) * 1e-3
    assert host_work > 0
    assert torch.equal(RRi, ref)
    # the call enqueues about 2 x 190 MB of copies: it must not have waited for them
    assert t_call < 0.5 * t_dev, (t_call, t_dev)
