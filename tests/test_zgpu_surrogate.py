"""Gated surrogate on the GPU: trained by the library's own BF16 kernels on
samples of the FP64 GPU integrator, applied through the conservation +
confidence gate with the FP64 integrator as fallback, and compared with a
plain FP64 integration of the same cells."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _element_mass(tables, Y):
    A = torch.tensor(tables.elem_matrix / tables.W[None, :], dtype=torch.float64, device=Y.device)
    return A @ Y          # [nel, n] kmol of each element per kg


def test_element_projector_conserves(small):
    from openhurricane_b200.surrogate import element_projector
    t = small["tables"]
    P = element_projector(t)
    A = t.elem_matrix / t.W[None, :]
    rng = np.random.default_rng(0)
    d = rng.normal(size=(t.nsp, 50))
    assert np.abs(A @ (P @ d)).max() < 1e-14 * np.abs(d).max()
    assert np.abs((P @ d).sum(axis=0)).max() < 1e-13 * np.abs(d).max()


def test_gated_surrogate_small_mechanism(small):
    from openhurricane_b200 import synth, workloads
    from openhurricane_b200.chemistry import ChemistrySource, Flow, Mechanism
    from openhurricane_b200.surrogate import Surrogate, generate_samples
    dev = torch.device("cuda:0")
    t = small["tables"]
    mech = Mechanism(t)
    opts = None
    from openhurricane_b200 import _capi
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)

    base = workloads.make_batched(16384, seed=77, pool=2048)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    s = generate_samples(mech, d(base.T), d(base.p), d(base.rho), d(base.Y), 1e-5, 131072,
                         seed=1, opts=opts)
    sur = Surrogate(mech, n_hidden=3, width=256, max_batch=65536, seed=2, n_ensemble=3)
    sur.fit_normalisation(s["T"], s["p"], s["Y"], s["dt"], s["dT"], s["dY"])
    X = sur.features(s["T"], s["p"], s["Y"], s["dt"])
    D = sur.targets(s["dT"], s["dY"])
    losses = sur.train(X, D, epochs=120, batch=8192, lr=2e-3)
    assert losses[-1] < 0.6 * losses[0]

    test = workloads.make_batched(32768, seed=99, pool=2048)
    n = test.n
    ref = Flow(d(test.T), d(test.p), d(test.rho), d(test.Y))
    dt = torch.full((n,), 1e-5, dtype=torch.float64, device=dev)
    # the method without the network: every cell by the FP64 integrator
    plain = ChemistrySource(mech, ref, **workloads.SOLVER_OPTS)
    plain.rebin = False
    plain.solveUpdate(dt, 1.0, counters=True)
    flow = Flow(d(test.T), d(test.p), d(test.rho), d(test.Y))
    e0 = _element_mass(t, flow.Y)
    fallback = {}
    nrej, accept = sur.step(flow, dt, opts=opts, counters=fallback)
    torch.cuda.synchronize()
    acc = accept.bool()
    dT = (flow.T - ref.T).abs()
    # what the network gains: the FP64 Newton iterations (each a Jacobian, an
    # LU and a solve) the gated step leaves to the integrator, against the
    # plain step's on the same cells
    gain = plain.last_counters["n_newton"] / max(1, fallback["n_newton"])
    print(f"rejected {nrej}/{n}, max|dT| accepted {dT[acc].max().item():.3f} K, "
          f"FP64 work of the plain step / of the gated step's fallback = {gain:.2f}")
    assert nrej < n                     # the network takes part
    assert gain > 1.5
    assert dT.max().item() < 5.0
    # rejected cells: the FP64 integrator's own result
    assert torch.equal(flow.T[~acc], ref.T[~acc])
    e1 = _element_mass(t, flow.Y)
    rel = ((e1 - e0).abs() / e0.abs().max(dim=0, keepdim=True).values)[:, acc]
    assert rel.max().item() < 1e-10
