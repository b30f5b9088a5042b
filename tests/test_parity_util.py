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
