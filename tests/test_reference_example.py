"""The reader and the oracle on the reference's own example mechanism (the
9-species / 19-reaction H2/air set of its ObliqueDetonation case, read in
place from the reference tree), against the reference compiled from its
sources: the tables must drive the oracle to the reference's answers bit
for bit through an ignition. Skipped where the reference tree or its build
is absent (the files are not copied into this repository)."""
import os
import tempfile

import numpy as np
import pytest

# the reference tree: HC_REFERENCE, else the Makefile's default (oracle/Makefile.ref)
EXAMPLE = os.path.join(os.environ.get("HC_REFERENCE", "/root/reference"), "example", "ObliqueDetonation")


def _files():
    f = (os.path.join(EXAMPLE, "in_mechanism.che"), os.path.join(EXAMPLE, "thermo7.dat"),
         os.path.join(EXAMPLE, "transport.dat"))
    if not all(os.path.isfile(x) for x in f):
        pytest.skip("reference example mechanism not present")
    return f


def _stoichiometric_h2_air(t, n, T_lo, T_hi):
    names, W = t.names, t.W
    x = {"H2": 2.0, "O2": 1.0, "N2": 3.76}
    tot = sum(v * W[names.index(k)] for k, v in x.items())
    Y = np.zeros((t.nsp, n))
    for k, v in x.items():
        Y[names.index(k)] = v * W[names.index(k)] / tot
    T = np.linspace(T_lo, T_hi, n)
    p = np.full(n, 101325.0)
    from openhurricane_b200 import mechanism
    rho = p / ((Y / W[:, None]).sum(axis=0) * mechanism.RU * T)
    return T, p, rho, Y


def test_example_mechanism_ignition_matches_the_reference():
    from openhurricane_b200 import mechanism
    from oracle import port, refrun
    files = _files()
    if not refrun.available():
        pytest.skip("reference binary not built (make -f oracle/Makefile.ref)")
    t = mechanism.compile_mechanism(*files)
    assert (t.nsp, t.nrc) == (9, 19)
    work = tempfile.mkdtemp()
    case = os.path.join(work, "case.cont")
    refrun.write_case(case, *files, {"atol": 1e-15})
    T, p, rho, Y = _stoichiometric_h2_air(t, 6, 1100.0, 1400.0)
    r = refrun.integrate(case, T, p, rho, 2e-4, 2e-4, Y, procs=4, workdir=work)
    o = port.integrate(port.MechDesc(t), T, p, rho, Y, 2e-4, subdt=2e-4,
                       opts=port.default_opts(atol=1e-15))
    for k in ("T", "Y", "rho", "c", "subdt"):
        assert np.array_equal(o[k], r[k]), k
    assert (o["T"] > 2500.0).all()          # every cell ignited within the step


def test_example_mechanism_known_answers_match_the_reference():
    from openhurricane_b200 import mechanism
    from oracle import port, refrun
    files = _files()
    if not refrun.available():
        pytest.skip("reference binary not built (make -f oracle/Makefile.ref)")
    t = mechanism.compile_mechanism(*files)
    work = tempfile.mkdtemp()
    case = os.path.join(work, "case.cont")
    refrun.write_case(case, *files, {"atol": 1e-15})
    rng = np.random.default_rng(31)
    n = 6
    T = rng.uniform(800.0, 3000.0, n)
    p = rng.uniform(1.0, 5.0, n) * 101325.0
    c = rng.dirichlet(np.full(t.nsp, 0.5), n).T.copy() * rng.uniform(0.001, 0.1, n)
    k = refrun.kat(case, p, T, c, workdir=work)
    dydt, J = port.rhs_jac(port.MechDesc(t), c, T, p)
    assert np.array_equal(dydt, k["dydt"])
    assert np.array_equal(J, k["J"])


def test_named_third_body_falloff_matches_the_reference(small, tmp_path):
    """A fall-off reaction with a named third body, (+N2): efficiency 1 for N2
    and 0 for the others (chemkinFileRead.cpp:1002-1061), through the reader
    and the oracle against the reference build."""
    from openhurricane_b200 import mechanism, synth
    from oracle import port, refrun
    if not refrun.available():
        pytest.skip("reference binary not built (make -f oracle/Makefile.ref)")
    che, th, tr = small["files"]
    txt = open(che).read()
    assert "(+M)" in txt
    # the reaction's efficiency line is dropped: with a named third body the
    # reference takes an efficiency for that species only
    lines, out, skip = txt.replace("(+M)", "(+N2)").splitlines(), [], False
    for line in lines:
        if "(+N2)" in line:
            skip = True
        elif skip and "/" in line and not line.strip().upper().startswith(("LOW", "TROE")):
            continue
        elif "=" in line:
            skip = False
        out.append(line)
    che2 = str(tmp_path / "named.che")
    with open(che2, "w") as f:
        f.write("\n".join(out) + "\n")
    t = mechanism.compile_mechanism(che2, th, tr)
    r = int(np.flatnonzero(t.rate_type >= mechanism.RATE_LINDEMANN)[0])
    assert t.eff[r, t.names.index("N2")] == 1.0 and t.eff[r].sum() == 1.0
    with pytest.raises(ValueError, match="third body"):
        with open(str(tmp_path / "bad.che"), "w") as f:
            f.write(txt.replace("(+M)", "(+N2)"))
        mechanism.compile_mechanism(str(tmp_path / "bad.che"), th, tr)
    case = str(tmp_path / "case.cont")
    refrun.write_case(case, che2, th, tr, {"atol": 1e-15})
    c = synth.dirichlet_cells(t.nsp, 8, seed=303)
    rho = synth.mixture_density(t.W, c)
    ref = refrun.integrate(case, c.T, c.p, rho, 1e-6, 1e-6, c.Y, procs=4, workdir=str(tmp_path))
    o = port.integrate(port.MechDesc(t), c.T, c.p, rho, c.Y, 1e-6,
                       opts=port.default_opts(atol=1e-15))
    for k in ("T", "Y", "rho", "c", "subdt"):
        assert np.array_equal(o[k], ref[k]), k


def _fitted_kat(t, case, tmp_path):
    """Known answers of the reference at six states against the oracle: DyDt,
    the Jacobian and kf / Kc / kr of every reaction, bit for bit."""
    from oracle import port, refrun
    rng = np.random.default_rng(3)
    T = rng.uniform(800.0, 3000.0, 6)
    p = rng.uniform(1.0, 5.0, 6) * 101325.0
    cc = rng.dirichlet(np.full(t.nsp, 0.5), 6).T.copy() * 0.01
    k = refrun.kat(case, p, T, cc, workdir=str(tmp_path))
    md = port.MechDesc(t)
    f, J = port.rhs_jac(md, cc, T, p)
    assert np.array_equal(f, k["dydt"]) and np.array_equal(J, k["J"])
    for s in range(6):
        r = port.rates(md, T[s], cc[:, s], p[s])
        assert np.array_equal(r[:, 0], k["kf"][s]) and np.array_equal(r[:, 2], k["kr"][s])


def test_collision_derivative_branch_matches_the_reference(tmp_path):
    """A collision-efficiency reaction with b != 0: the reference's dk/dT
    (Arrhenius derivative at k times dZ/dT) enters the Jacobian; known
    answers only (integrations with it stall, see synth.fitted_rates_mechanism)."""
    from oracle import refrun
    from openhurricane_b200 import mechanism, synth
    if not refrun.available():
        pytest.skip("reference binary not built (make -f oracle/Makefile.ref)")
    files = synth.write_chemkin(synth.fitted_rates_mechanism(collision=(1e-22, 0.5, 0.0)),
                                str(tmp_path / "m"))
    t = mechanism.compile_mechanism(*files)
    r = int(np.where(t.rate_type == mechanism.RATE_COLLISION)[0][0])
    assert t.arr[r, 1] == 0.5
    case = str(tmp_path / "case.cont")
    # a viscous flow model: the reference reads the transport data (the
    # collision diameters) only then, and dereferences an empty table otherwise
    refrun.write_case(case, *files, {"atol": 1e-15, "flowModel": "laminarFlow"})
    _fitted_kat(t, case, tmp_path)


def test_fitted_rates_match_the_reference(fitted, tmp_path):
    """Janev (JAN), power-series (FIT1), reverse Landau-Teller (RLT) and
    collision-efficiency (COLLEFF) rates: reader and oracle against the
    reference build, by integration and known answers."""
    from oracle import port, refrun
    if not refrun.available():
        pytest.skip("reference binary not built (make -f oracle/Makefile.ref)")
    t = fitted["tables"]
    assert sorted(set(t.rate_type) & {7, 8, 9, 10}) == [7, 8, 9, 10]
    case = str(tmp_path / "case.cont")
    refrun.write_case(case, *fitted["files"], {"atol": 1e-15, "flowModel": "laminarFlow"})
    from openhurricane_b200 import synth
    c = synth.dirichlet_cells(t.nsp, 12, seed=41)
    rho = synth.mixture_density(t.W, c)
    r = refrun.integrate(case, c.T, c.p, rho, 1e-6, 1e-6, c.Y, procs=4, workdir=str(tmp_path))
    md = port.MechDesc(t)
    o = port.integrate(md, c.T, c.p, rho, c.Y, 1e-6, opts=port.default_opts(atol=1e-15))
    for k in ("T", "Y", "rho", "c", "subdt"):
        assert np.array_equal(o[k], r[k]), k
    _fitted_kat(t, case, tmp_path)
