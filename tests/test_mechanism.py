"""Mechanism compiler (openhurricane_b200/mechanism.py): reference unit
conversions and table layout."""
import math

import numpy as np

from openhurricane_b200 import mechanism as M


def test_constants_match_reference_expressions():
    assert M.RU == (1.380649e-23 * 6.02214076e23) * 1e3
    assert M.PATM == 1.01325e5


def test_weights_and_mass_basis_nasa(small):
    t = small["tables"]
    m = small["mech"]
    for i, s in enumerate(m.species):
        w = 0.0
        for el in ("C", "H", "O", "N"):
            if el in s.elements:
                w += s.elements[el] * M.ATOMIC_WEIGHTS[el]
        assert t.W[i] == w
        assert t.Ri[i] == M.RU / w
    raw = float(f"{m.species[0].low[0]:15.8E}")
    assert t.nasa[0, 0, 0] == raw * t.Ri[0]


def test_reaction_tables(small):
    t = small["tables"]
    m = small["mech"]
    assert t.nrc == 21
    assert (t.rate_type == M.RATE_THIRD_BODY).sum() == 3
    assert (t.rate_type == M.RATE_TROE4).sum() == 1
    for r, rx in enumerate(m.reactions):
        names = [t.names[t.fidx[r, k]] for k in range(t.nf[r])]
        assert names == sorted(names)      # std::map order of the reference parser
        order = sum(n for _, n in rx.reactants)
        fac = math.pow(0.001, order - 1.0)
        A_file = float(f"{rx.A:.6E}")
        E_file = float(f"{rx.Ea:.4f}")
        if rx.kind == "third_body":
            assert t.arr[r, 0] == 1e-3 * A_file * fac
        else:
            assert t.arr[r, 0] == A_file * fac
        assert t.arr[r, 2] == E_file / (M.R_J_MOL_K / M.CAL_TH)
        assert t.sum_stoi[r] == t.bnu[r, :t.nb[r]].sum() - t.fnu[r, :t.nf[r]].sum()


def test_large_mechanism_shape_and_element_balance(large):
    t = large["tables"]
    assert t.nsp == 53 and t.nrc == 325
    assert (t.rate_type == M.RATE_THIRD_BODY).sum() == 49
    assert (t.rate_type == M.RATE_TROE4).sum() == 16
    E = t.elem_matrix
    for r in range(t.nrc):
        bal = np.zeros(E.shape[0])
        for k in range(t.nf[r]):
            bal -= t.fnu[r, k] * E[:, t.fidx[r, k]]
        for k in range(t.nb[r]):
            bal += t.bnu[r, k] * E[:, t.bidx[r, k]]
        assert np.all(bal == 0)
