"""The device state (hc_state_*): fields uploaded once, stepped on the
device, downloaded in either layout; against the pointer-based entry points
on the same cells, bit for bit (the same kernels run on the same numbers)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _dev():
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    return torch.device("cuda:0")


def _cells(tables, n, seed):
    from openhurricane_b200 import synth
    c = synth.dirichlet_cells(tables.nsp, n, seed=seed)
    return c.T, c.p, synth.mixture_density(tables.W, c), np.ascontiguousarray(c.Y)


def _h(a):
    return a.ctypes.data_as(C.c_void_p)


def test_state_step_matches_host_entry_point(small):
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = small["tables"]
    m = Mechanism(t)
    lib = _capi.load()
    n = 211
    T, p, rho, Y = _cells(t, n, seed=901)
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)
    dt = np.full(n, 1e-7)
    # pointer-based host entry point
    Th, rh, Yh, sub_h, Ri_h = T.copy(), rho.copy(), Y.copy(), dt.copy(), np.zeros_like(Y)
    st_h = np.zeros(n, np.int32)
    assert lib.hc_integrate_host(m.handle, C.byref(opts), n, _h(Th), _h(p), _h(rh), _h(Yh), _h(dt),
                                 1.0, _h(sub_h), _h(Ri_h), _h(st_h), None, None) >= 0
    # the device state
    s = C.c_void_p()
    _capi.check(lib.hc_state_create(m.handle, n, C.byref(s)), "hc_state_create")
    try:
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _capi.check(lib.hc_upload(s, _h(T), _h(p), _h(rho), _h(Y), None, stream), "hc_upload")
        dt_d = torch.tensor(dt, device=dev)
        _capi.check(lib.hc_state_integrate(s, C.byref(opts), C.c_void_p(dt_d.data_ptr()), 1.0,
                                           stream), "hc_state_integrate")
        To, ro, Yo, Rio, so = (np.zeros(n), np.zeros(n), np.zeros_like(Y), np.zeros_like(Y),
                               np.zeros(n))
        sto = np.zeros(n, np.int32)
        _capi.check(lib.hc_download(s, _h(To), _h(ro), _h(Yo), _h(Rio), _h(so), _h(sto), stream),
                    "hc_download")
        assert np.array_equal(To, Th) and np.array_equal(ro, rh) and np.array_equal(Yo, Yh)
        assert np.array_equal(Rio, Ri_h) and np.array_equal(so, sub_h)
        assert np.array_equal(sto, st_h)
        # a second step starts from the warm sub-steps the first one left
        _capi.check(lib.hc_state_integrate(s, C.byref(opts), C.c_void_p(dt_d.data_ptr()), 1.0,
                                           stream), "hc_state_integrate")
        _capi.check(lib.hc_download(s, _h(To), None, None, None, None, None, stream), "hc_download")
        assert np.all(np.isfinite(To))
    finally:
        lib.hc_state_destroy(s)


def test_state_records_and_evaluations(large):
    from openhurricane_b200 import _capi
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = large["tables"]
    m = Mechanism(t)
    lib = _capi.load()
    n = 301
    T, p, rho, Y = _cells(t, n, seed=902)
    s = C.c_void_p()
    _capi.check(lib.hc_state_create(m.handle, n, C.byref(s)), "hc_state_create")
    try:
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        # [T, Y..., rho] records with the caller's p
        rec = np.ascontiguousarray(np.concatenate([T[:, None], Y.T, rho[:, None]], axis=1))
        _capi.check(lib.hc_upload_records(s, 0, _h(rec), _h(p), stream), "hc_upload_records")
        To, ro, Yo = np.zeros(n), np.zeros(n), np.zeros_like(Y)
        _capi.check(lib.hc_download(s, _h(To), _h(ro), _h(Yo), None, None, None, stream),
                    "hc_download")
        assert np.array_equal(To, T) and np.array_equal(ro, rho) and np.array_equal(Yo, Y)
        out = np.zeros((n, t.nsp + 2))
        _capi.check(lib.hc_download_records(s, 1, _h(out), stream), "hc_download_records")
        assert np.array_equal(out, np.concatenate([Y.T, rho[:, None], T[:, None]], axis=1))
        # source terms and properties at the state's fields
        d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
        Ri_ref = m.source_terms(d(T), d(p), d(rho), d(Y)).cpu().numpy()
        _capi.check(lib.hc_state_source_terms(s, stream), "hc_state_source_terms")
        Rio = np.zeros_like(Y)
        _capi.check(lib.hc_download(s, None, None, None, _h(Rio), None, None, stream), "hc_download")
        assert np.array_equal(Rio, Ri_ref)
        ref = m.properties(d(T), d(p), d(Y))
        cp = torch.empty(n, dtype=torch.float64, device=dev)
        mu = torch.empty(n, dtype=torch.float64, device=dev)
        _capi.check(lib.hc_state_properties(s, None, C.c_void_p(cp.data_ptr()),
                                            C.c_void_p(mu.data_ptr()), None, None, stream),
                    "hc_state_properties")
        torch.cuda.synchronize()
        assert torch.equal(cp, ref["cp"]) and torch.equal(mu, ref["mu"])
        # [Y..., T, p] records carry p: the diffusion coefficients (1/p) follow it
        rec2 = np.ascontiguousarray(np.concatenate([Y.T, T[:, None], (p * 2.0)[:, None]], axis=1))
        _capi.check(lib.hc_upload_records(s, 2, _h(rec2), None, stream), "hc_upload_records")
        D = torch.empty((t.nsp, n), dtype=torch.float64, device=dev)
        _capi.check(lib.hc_state_properties(s, None, None, None, None, C.c_void_p(D.data_ptr()),
                                            stream), "hc_state_properties")
        torch.cuda.synchronize()
        assert torch.equal(D, m.properties(d(T), d(p * 2.0), d(Y))["D"])
        pp = C.c_void_p()
        _capi.check(lib.hc_state_fields(s, None, C.byref(pp), None, None, None, None, None),
                    "hc_state_fields")
        assert pp.value is not None
    finally:
        lib.hc_state_destroy(s)


def test_property_records_match_species_major_fields(large):
    """calchaicp / calcTransportProperties records ([Y..., T, p] in;
    [h..., cp] and [D..., mu, kappa] out) against hc_properties on the same
    cells, device and host forms, bit for bit."""
    from openhurricane_b200 import _capi
    from openhurricane_b200.chemistry import Mechanism
    dev = _dev()
    t = large["tables"]
    m = Mechanism(t)
    n = 1037
    T, p, rho, Y = _cells(t, n, seed=816)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    ref = m.properties(d(T), d(p), d(Y))
    rec = np.ascontiguousarray(np.concatenate([Y.T, T[:, None], p[:, None]], axis=1))
    hc = torch.empty((n, t.nsp + 1), dtype=torch.float64, device=dev)
    dmk = torch.empty((n, t.nsp + 2), dtype=torch.float64, device=dev)
    vp = lambda x: C.c_void_p(x.data_ptr())
    lib = _capi.load()
    rec_d = d(rec)
    assert lib.hc_properties_aos(m.handle, n, vp(rec_d), vp(hc), vp(dmk),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    hc, dmk = hc.cpu().numpy(), dmk.cpu().numpy()
    assert np.array_equal(hc[:, :-1], ref["ha"].cpu().numpy().T)
    assert np.array_equal(hc[:, -1], ref["cp"].cpu().numpy())
    assert np.array_equal(dmk[:, :-2], ref["D"].cpu().numpy().T)
    assert np.array_equal(dmk[:, -2], ref["mu"].cpu().numpy())
    assert np.array_equal(dmk[:, -1], ref["kappa"].cpu().numpy())
    hc_h = np.zeros((n, t.nsp + 1))
    assert lib.hc_properties_aos_host(m.handle, n, rec.ctypes.data_as(C.c_void_p),
                                      hc_h.ctypes.data_as(C.c_void_p), None, None) == 0
    assert np.array_equal(hc_h, hc)
