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


def test_unit_factors_follow_the_reference_change_unit():
    """chemkinFileRead::changeUnit: A from [mol or molecule, cm^3, s] to
    [kmol, m^3, s], E to an activation temperature."""
    R = M.R_J_MOL_K
    for order in (1.0, 1.5, 2.0, 3.0):
        Af, Ef = M.change_unit(order, "MOLES", "CAL", False)
        assert Af == math.pow(0.001, order - 1.0) and Ef == R / M.CAL_TH
        Af, _ = M.change_unit(order, "MOLECULES", "CAL", False)
        assert Af == math.pow(M.NA, order - 1.0) * math.pow(0.001, order - 1.0)
        Af, _ = M.change_unit(order, "MOLECULES", "CAL", True)
        assert Af == math.pow(M.NA, order) * math.pow(0.001, order - 1.0)
    E = {u: M.change_unit(2.0, "MOLES", u, False)[1]
         for u in ("CAL", "KCAL", "JOUL", "KJOU", "KELV", "EVOL")}
    assert E["KCAL"] == (R / M.CAL_TH) / 1000.0 and E["JOUL"] == R
    assert E["KJOU"] == R / 1000.0 and E["KELV"] == 1.0 and E["EVOL"] == R / M.ELECTRON_VOLT


def test_extended_rate_forms_are_read(ext):
    t = ext["tables"]
    m = ext["mech"]
    assert m.units == ("KJOU", "MOLES")
    sri = np.flatnonzero(t.rate_type == M.RATE_SRI)
    assert len(sri) == 2
    five = [r for r in m.reactions if r.sri is not None and len(r.sri) == 5][0]
    three = [r for r in m.reactions if r.sri is not None and len(r.sri) == 3][0]
    rows = {tuple(t.sri[r, :3]) for r in sri}
    assert tuple(three.sri) in rows and tuple(five.sri[:3]) in rows
    for r in sri:
        if tuple(t.sri[r, :3]) == tuple(three.sri):
            assert t.sri[r, 3] == 1.0 and t.sri[r, 4] == 0.0      # SRI(a, b, c): d = 1, e = 0
        else:
            assert tuple(t.sri[r]) == tuple(five.sri)
    rev = np.flatnonzero(t.reversible == M.REVERSIBLE_REV)
    assert len(rev) == 3
    assert set(t.rate_type[rev]) == {M.RATE_ARRHENIUS, M.RATE_THIRD_BODY}
    assert (t.arr_rev[rev, 0] > 0).all() and (t.arr_rev[t.reversible != 2] == 0).all()
    # one chemically activated reaction (HIGH, here with the 5-parameter SRI form):
    # k0 from its main line (A factor 1e-3 for order 2), kinf from HIGH (x 1e3)
    act = np.flatnonzero(t.activated)
    assert len(act) == 1 and t.rate_type[act[0]] == M.RATE_SRI
    hi = [r for r in m.reactions if r.activated][0]
    assert np.isclose(t.arr0[act[0], 0], hi.low[0] * 1e-3, rtol=1e-6)
    assert np.isclose(t.arr[act[0], 0], hi.A * 1e-3 / 1e-3, rtol=1e-6)
    ltr = np.flatnonzero(t.rate_type == M.RATE_LANDAU_TELLER)
    assert len(ltr) == 1 and tuple(t.lt[ltr[0]]) == [r for r in m.reactions if r.lt][0].lt
    # the FORD / RORD overrides change the order only, not the stoichiometry
    assert (t.ford != t.fnu).sum() == 1 and t.ford[t.ford != t.fnu][0] == 1.5
    assert (t.bord != t.bnu).sum() == 1 and t.bord[t.bord != t.bnu][0] == 1.5


def test_energy_units_give_the_same_activation_temperature(tmp_path):
    """The same reaction written with E in cal/mol, kcal/mol, kJ/mol and K
    (REACTIONS-line and per-reaction units) reads to one activation
    temperature, to the digits printed (four decimals of kcal/mol are 0.05 K)."""
    from openhurricane_b200 import synth
    base = synth.small_mechanism()
    che, th, tr = synth.write_chemkin(base, str(tmp_path / "a"))
    t0 = M.compile_mechanism(che, th, tr)
    for units, per in ((("KCAL",), None), (("KJOU", "MOLES"), None), ((), "KELV")):
        m = synth.small_mechanism()
        m.units = units
        if per:
            for r in m.reactions:
                r.units = per
        che, th, tr = synth.write_chemkin(m, str(tmp_path / ("u" + "".join(units) + (per or ""))))
        t = M.compile_mechanism(che, th, tr)
        assert np.allclose(t.arr[:, 2], t0.arr[:, 2], rtol=0.0, atol=0.06)
        assert np.array_equal(t.arr[:, 0], t0.arr[:, 0])


def _che(body, header="REACTIONS"):
    return ("ELEMENTS\nH O\nEND\nSPECIES\nH2 O2 H O HO\nEND\n" + header + "\n" + body + "\nEND\n")


def test_reader_rejects_what_it_does_not_take():
    import pytest
    with pytest.raises(NotImplementedError, match="CHEB"):
        M.parse_chemkin(_che("H2+O2=2HO 1.0E13 0.0 1000.0\n CHEB / 7 4 /"))
    with pytest.raises(ValueError, match="PLOG"):
        M.parse_chemkin(_che("H2+O2+M=2HO+M 1.0E13 0.0 1000.0\n PLOG / 1.0 1.0E13 0.0 1000.0 /"))
    with pytest.raises(ValueError, match="FORD"):
        M.parse_chemkin(_che("H2+O2=2HO 1.0E13 0.0 1000.0\n FORD / O 0.5 /"))
    with pytest.raises(ValueError, match="unit"):
        M.parse_chemkin(_che("H2+O2=2HO 1.0E13 0.0 1000.0", header="REACTIONS FURLONGS"))
    names, _, rx = M.parse_chemkin(_che(
        "H+O2(+M)=HO+O(+M) 1.0E13 0.0 1000.0\n LOW / 1.0E16 0.0 0.0 /\n REV / 1.0E12 0.0 0.0 /"))
    assert rx[0].rev is not None and rx[0].kind == "falloff"


def test_plog_tables_are_sorted_and_converted(ext, tmp_path):
    """PLOG entries sorted by pressure (equal pressures in file order), in Pa,
    with the reaction's A and E factors; a repeated highest pressure is
    refused (the reference's derivative reads past its table there)."""
    import pytest
    t = ext["tables"]
    rows = np.flatnonzero(t.rate_type == M.RATE_PLOG)
    assert len(rows) == 3 and t.plog_ptr[-1] == 9
    for r in rows:
        pp = t.plog_p[t.plog_ptr[r]:t.plog_ptr[r + 1]]
        assert (np.diff(pp) >= 0).all() and pp[-1] > pp[-2]
    assert set(np.round(t.plog_p / M.PATM, 6)) == {0.01, 0.1, 0.5, 1.0, 10.0, 100.0}
    src = [r for r in ext["mech"].reactions if r.plog]
    dup = [r for r in src if r.plog[0][0] == r.plog[1][0]][0]
    r = [i for i in rows if t.plog_p[t.plog_ptr[i]] == t.plog_p[t.plog_ptr[i] + 1]][0]
    b = t.plog_ptr[r]
    # file order kept for the equal pressures; A in kmol-m-s (order 2: x 1e-3)
    assert np.allclose(t.plog_arr[b:b + 2, 0], [dup.plog[0][1] * 1e-3, dup.plog[1][1] * 1e-3],
                       rtol=1e-6)
    che = _che("H2+O2=2HO 1.0E13 0.0 1000.0\n PLOG / 1.0 1.0E13 0.0 1000.0 /\n"
               " PLOG / 1.0 2.0E13 0.0 1000.0 /")
    names, els, rx = M.parse_chemkin(che)
    assert len(rx[0].plog) == 2
    f = tmp_path / "m.che"
    f.write_text(che)
    with pytest.raises(ValueError, match="highest pressure"):
        M.compile_mechanism(str(f), *ext["files"][1:])


def test_thermo_and_transport_sections_in_the_mechanism_file(small, tmp_path):
    """Without separate files, the THERMO and TRANSPORT sections of the
    mechanism file are read (as the reference's reader does) and give the same
    tables."""
    che, th, tr = small["files"]
    txt = open(che).read() + "\nTHERMO\n" + open(th).read().split("THERMO", 1)[1] + \
        "\nTRANSPORT\n" + open(tr).read() + "END\n"
    one = tmp_path / "all_in_one.che"
    one.write_text(txt)
    a = small["tables"]
    b = M.compile_mechanism(str(one))
    for k in ("W", "nasa", "Trange", "arr", "arr0", "troe", "eff", "geom", "eps_k", "sigma"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_janev_and_power_series_tables(fitted):
    """JAN keeps A, beta and Ta of the main line and 9 coefficients; FIT1 keeps
    A and beta (its E is not used) and 4 coefficients in the first columns."""
    t = fitted["tables"]
    m = fitted["mech"]
    rx = m.reactions
    j = next(i for i, r in enumerate(rx) if r.janev is not None)
    f = next(i for i, r in enumerate(rx) if r.fit1 is not None)
    assert t.rate_type[j] == M.RATE_JANEV and t.rate_type[f] == M.RATE_POWER_SERIES
    assert np.array_equal(t.xcoef[j], np.array(rx[j].janev))
    assert np.array_equal(t.xcoef[f, :4], np.array(rx[f].fit1))
    assert not t.xcoef[f, 4:].any()
    assert t.arr[f, 2] == 0.0 and t.arr[j, 2] > 0.0
    others = [i for i in range(len(rx)) if i not in (j, f) and rx[i].rlt is None
              and not rx[i].collision]
    assert not t.xcoef[others].any()
    import pytest
    with pytest.raises(ValueError, match="JAN"):
        M.parse_chemkin(_che("H2+O2(+M)=2HO(+M) 1.0E13 0.0 1000.0\n LOW / 1.0E16 0.0 0.0 /\n"
                             " JAN / 1 2 3 4 5 6 7 8 9 /"))
    with pytest.raises(ValueError, match="FIT1 takes 4"):
        M.parse_chemkin(_che("H2+O2=2HO 1.0E13 0.0 1000.0\n FIT1 / 1 2 3 /"))


def test_reverse_landau_teller_tables(fitted):
    """LT + REV + RLT: the reverse rate takes REV's A, beta, Ta and RLT's B, C
    (in xcoef); RLT needs REV before it and LT on the reaction."""
    t = fitted["tables"]
    rx = fitted["mech"].reactions
    k = next(i for i, r in enumerate(rx) if r.rlt is not None)
    assert t.rate_type[k] == M.RATE_LANDAU_TELLER and t.reversible[k] == M.REVERSIBLE_REV
    assert np.array_equal(t.lt[k], np.array(rx[k].lt))
    assert np.array_equal(t.xcoef[k, :2], np.array(rx[k].rlt)) and not t.xcoef[k, 2:].any()
    assert t.arr_rev[k, 1] == rx[k].rev[1]
    import pytest
    with pytest.raises(ValueError, match="must follow the explicit REV"):
        M.parse_chemkin(_che("H2+O2=2HO 1.0E13 0.0 1000.0\n LT / 1 2 /\n RLT / 1 2 /\n"
                             " REV / 1.0E12 0.0 0.0 /"))
    with pytest.raises(ValueError, match="RLT on a reaction without LT"):
        M.compile_mechanism(*_without(fitted, "   LT / "))
    with pytest.raises(ValueError, match="needs RLT"):
        M.compile_mechanism(*_without(fitted, "   RLT / "))


def _without(fixture, prefix):
    """The fixture's files with the mechanism lines that start with `prefix` dropped."""
    import os
    import tempfile
    che, th, tr = fixture["files"]
    d = tempfile.mkdtemp()
    text = open(che).read().splitlines()
    text = [l for l in text if not l.startswith(prefix)]
    out = os.path.join(d, "chem.inp")
    with open(out, "w") as f:
        f.write("\n".join(text) + "\n")
    return out, th, tr


def test_collision_efficiency_tables(fitted):
    """COLLEFF: the main line is the efficiency; xcoef holds N_A d^2 and
    8 pi / 2 pi times Ru / W_AB, d the mean collision diameter of the two
    reactants as read (angstrom), W_AB their reduced molar mass."""
    t = fitted["tables"]
    rx = fitted["mech"].reactions
    k = next(i for i, r in enumerate(rx) if r.collision)
    assert t.rate_type[k] == M.RATE_COLLISION and t.reversible[k] == M.REVERSIBLE
    (a, _), (b, _) = ((t.names.index(n), v) for n, v in rx[k].reactants)
    d = (t.sigma[a] + t.sigma[b]) / 2.0
    wab = t.W[a] * t.W[b] / (t.W[a] + t.W[b])
    assert math.isclose(t.xcoef[k, 0], M.NA * d * d, rel_tol=1e-15)
    assert math.isclose(t.xcoef[k, 1], 8.0 * math.pi * M.RU / wab, rel_tol=1e-15)
    assert math.isclose(t.xcoef[k, 2], 2.0 * math.pi * M.RU / wab, rel_tol=1e-15)
    assert not t.xcoef[k, 3:].any()
    import pytest
    with pytest.raises(ValueError, match="bimolecular"):
        M.parse_chemkin(_che("H2+O2+HO=2HO+H 1.0E13 0.0 1000.0\n COLLEFF"))
    with pytest.raises(ValueError, match="third-body or fall-off"):
        M.parse_chemkin(_che("H2+O2+M=2HO+M 1.0E13 0.0 1000.0\n COLLEFF"))


def test_forms_the_reference_refuses_are_refused():
    import pytest
    for key in ("TDEP / H2 /", "XSMI / 1.0 /", "MOME / 1.0 /", "EXCI / 1.0 /"):
        with pytest.raises(NotImplementedError, match="not supported"):
            M.parse_chemkin(_che("H2+O2=2HO 1.0E13 0.0 1000.0\n " + key))
