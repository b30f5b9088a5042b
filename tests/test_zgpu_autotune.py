"""The launch-shape autotuner on the GPU: it times its candidates on a
sample of the caller's cells, applies the fastest, and the tuned launch
still gives the oracle's answer."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_autotune_picks_and_applies_a_working_shape(small):
    from openhurricane_b200 import autotune, synth
    from openhurricane_b200.chemistry import ChemistrySource, Flow, Mechanism
    from oracle import port
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    dev = torch.device("cuda:0")
    t = small["tables"]
    c = synth.dirichlet_cells(t.nsp, 512, seed=404)
    rho = synth.mixture_density(t.W, c)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    T, p, r, Y = d(c.T), d(c.p), d(rho), d(c.Y)
    dt = torch.full((512,), 1e-7, dtype=torch.float64, device=dev)
    m = Mechanism(t)
    res = autotune.autotune(m, T, p, r, Y, dt, sample=256, repeats=1,
                            cands=[(2, 64), (4, 64), (1, 64)])
    assert res["kernel"] in (1, 2, 4) and len(res["trials"]) == 3
    assert all(tr["ms"] > 0 for tr in res["trials"])
    flow = Flow(T.clone(), p, r.clone(), Y.clone())
    ChemistrySource(m, flow, atol=1e-15, rtol=1e-6).solveUpdate(dt)
    o = port.integrate(port.MechDesc(t), c.T, c.p, rho, c.Y, 1e-7,
                       opts=port.default_opts(atol=1e-15, rtol=1e-6))
    assert np.max(np.abs(flow.T.cpu().numpy() - o["T"]) / o["T"]) <= 1e-6


def test_entry_points_accept_zero_cells(small):
    from openhurricane_b200.chemistry import Mechanism
    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for -m gpu tests")
    dev = torch.device("cuda:0")
    nsp = small["tables"].nsp
    m = Mechanism(small["tables"])
    e = torch.zeros(0, dtype=torch.float64, device=dev)
    Y = torch.zeros((nsp, 0), dtype=torch.float64, device=dev)
    assert m.source_terms(e, e, e, Y).shape == (nsp, 0)
    Ri, diag = m.source_terms_imp(e, e, e, Y)
    assert Ri.shape == (nsp, 0) and diag.shape == (nsp - 1, 0)
    assert m.properties(e, e, Y)["mu"].shape == (0,)
    T, f = m.temperature_from_enthalpy(e, Y, e)
    assert T.shape == (0,)
