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

EXAMPLE = "/root/reference/example/ObliqueDetonation"


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
