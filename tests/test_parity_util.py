"""The parity helpers of the GPU tests (tests/parity_util.py), on the CPU:
answers equal to the oracle's pass, an answer the oracle reaches from a
one-ulp input perturbation is explained, and a planted error (in an
oracle answer standing in for the GPU's) is neither."""
import numpy as np
import pytest

import parity_util as pu


def _case(small, n=24, seed=31):
    from openhurricane_b200 import synth
    t = small["tables"]
    c = synth.dirichlet_cells(t.nsp, n, seed=seed)
    rho = synth.mixture_density(t.W, c)
    return t, (c.T, c.p, rho, c.Y)


def test_identical_answers_pass(small):
    t, inp = _case(small)
    o = pu.oracle(t, *inp, 1e-6, atol=1e-15)
    assert pu.bad_cells(o, o).size == 0
    pu.check(t, inp, o, o, 1e-6, dict(atol=1e-15), "identical")


def test_perturbed_start_is_explained(small):
    t, inp = _case(small)
    T, p, rho, Y = inp
    ref = pu.oracle(t, *inp, 1e-6, atol=1e-15)
    # the "GPU" answer: the oracle from inputs one ulp away (the first
    # perturbation explain() tries); where it left the tolerance, explain()
    # must reproduce it
    Tk, Yk = pu.perturbations(T, Y, 0)
    g = pu.oracle(t, Tk, p, rho, Yk, 1e-6, atol=1e-15)
    bad = pu.bad_cells(g, ref)
    left = pu.explain(t, inp, g, bad, 1e-6, dict(atol=1e-15)) if bad.size else bad
    assert left.size == 0


def test_planted_error_is_not_explained(small):
    t, inp = _case(small)
    ref = pu.oracle(t, *inp, 1e-7, atol=1e-15)
    g = {k: np.array(v, copy=True) for k, v in ref.items()}
    g["T"][5] *= 1.0 + 1e-4      # a wrong temperature in one cell
    bad = pu.bad_cells(g, ref)
    assert bad.tolist() == [5]
    assert pu.explain(t, inp, g, bad, 1e-7, dict(atol=1e-15), tries=4).tolist() == [5]
    with pytest.raises(AssertionError):
        pu.check(t, inp, g, ref, 1e-7, dict(atol=1e-15), "planted")


def test_reference_answers_on_indistinguishable_inputs_are_explained(small):
    """The criterion's calibration, on the benchmarked cells at the bench's
    options: oracle answers from one-ulp perturbations outside explain()'s
    own tries (the reference's algorithm on inputs indistinguishable from the
    cells' own) stand in for the GPU's answer, and every one of their cells
    outside the tolerance is explained."""
    import os
    g0 = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "batched_ref.npz"))
    t = small["tables"]
    inp = (g0["in_T"], g0["in_p"], g0["in_rho"], g0["in_Y"])
    dt = float(g0["dt"])
    opts = dict(atol=1e-11, rtol=1e-4)
    ref = {"T": g0["out_T"], "rho": g0["out_rho"], "Y": g0["out_Y"]}
    for k in (1017, 1023):
        Tk, Yk = pu.perturbations(inp[0], inp[3], k)
        g = pu.oracle(t, Tk, inp[1], inp[2], Yk, dt, **opts)
        bad = pu.bad_cells(g, ref)
        assert bad.size > 0      # the sample has cells that one ulp moves
        assert pu.explain(t, inp, g, bad, dt, opts, ref=ref).size == 0
