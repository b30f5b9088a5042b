"""The oracle (oracle/chem_oracle.c, oracle/props_oracle.py) is pinned to the
reference.

1. Against the committed golden fixtures, which the reference itself
   produced (tests/golden/make_golden.py): bit-for-bit equality of the
   integrated states and of the kernel-level known answers (DyDt, analytic
   Jacobian, NASA-7 thermo, kf/Kc/kr); properties within 1e-15 relative.
2. Against the reference compiled from source here (oracle/_ref/hurchem_ref),
   when that binary is present, on freshly drawn cells.
"""
import hashlib
import os
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _sha(paths):
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _load(name):
    return np.load(os.path.join(HERE, "golden", f"{name}_ref.npz"))


@pytest.mark.parametrize("name", ["small", "large", "ext", "fitted"])
def test_generator_reproduces_golden_mechanism(name, request):
    mk = request.getfixturevalue(name)
    assert _sha(mk["files"]) == str(_load(name)["sha"])


@pytest.mark.parametrize("name", ["small", "large", "ext", "fitted"])
def test_oracle_integration_bit_exact_vs_reference_golden(name, request):
    from oracle import port
    mk = request.getfixturevalue(name)
    g = _load(name)
    md = port.MechDesc(mk["tables"])
    o = port.integrate(md, g["in_T"], g["in_p"], g["in_rho"], g["in_Y"], float(g["dt"]),
                       opts=port.default_opts(atol=1e-15))
    for k in ("T", "Y", "rho", "c", "subdt"):
        assert np.array_equal(o[k], g["out_" + k]), k


@pytest.mark.parametrize("name,mech,opts", [
    ("batched", "small", dict(atol=1e-11, rtol=1e-4)),   # the benchmarked configuration
    ("large32", "large", dict(atol=1e-15)),
])
def test_oracle_integration_bit_exact_vs_reference_golden_at_options(name, mech, opts, request):
    """The benchmarked cells at the benchmark's solver options and 32 cells of
    the 53-species mechanism: the oracle reproduces the reference bit for bit."""
    from oracle import port
    mk = request.getfixturevalue(mech)
    g = _load(name)
    assert _sha(mk["files"]) == str(g["sha"])
    md = port.MechDesc(mk["tables"])
    o = port.integrate(md, g["in_T"], g["in_p"], g["in_rho"], g["in_Y"], float(g["dt"]),
                       opts=port.default_opts(**opts))
    for k in ("T", "Y", "rho", "c", "subdt"):
        assert np.array_equal(o[k], g["out_" + k]), k


@pytest.mark.parametrize("name", ["small", "large", "ext", "fitted"])
def test_oracle_kernels_bit_exact_vs_reference_golden(name, request):
    from oracle import port
    mk = request.getfixturevalue(name)
    g = _load(name)
    md = port.MechDesc(mk["tables"])
    dydt, J = port.rhs_jac(md, g["kat_c"], g["kat_T"], g["kat_p"])
    assert np.array_equal(dydt, g["kat_dydt"])
    assert np.array_equal(J, g["kat_J"])
    for s in range(g["kat_T"].shape[0]):
        assert np.array_equal(port.thermo(md, g["kat_T"][s]), g["kat_thermo"][s])
        assert np.array_equal(port.rates(md, g["kat_T"][s], g["kat_c"][:, s], g["kat_p"][s]),
                              g["kat_rates"][s])


@pytest.mark.parametrize("name", ["small", "large", "ext", "fitted"])
def test_property_oracle_vs_reference_golden(name, request):
    from oracle import props_oracle
    mk = request.getfixturevalue(name)
    g = _load(name)
    o = props_oracle.properties(mk["tables"], g["prop_T"], g["prop_p"], g["prop_Y"])
    for k in ("ha", "cp", "mu", "kappa", "D"):
        ref = g["prop_" + k]
        assert np.max(np.abs(o[k] - ref) / np.maximum(np.abs(ref), 1e-300)) < 1e-15, k


def test_oracle_bit_exact_vs_reference_binary(small):
    from oracle import refrun, port
    from openhurricane_b200 import synth
    if not refrun.available():
        pytest.skip("reference binary not built (make -f oracle/Makefile.ref)")
    t = small["tables"]
    work = tempfile.mkdtemp()
    case = os.path.join(work, "case.cont")
    refrun.write_case(case, *small["files"], {"atol": 1e-15, "rtol": 1e-5})
    cells = synth.dirichlet_cells(t.nsp, 12, seed=2024)
    cells.T[0] = 150.0      # below the 200 K threshold: skipped, dtInit = dt
    rho = synth.mixture_density(t.W, cells)
    r = refrun.integrate(case, cells.T, cells.p, rho, 1e-6, 5e-7, cells.Y, procs=4, workdir=work)
    o = port.integrate(port.MechDesc(t), cells.T, cells.p, rho, cells.Y, 1e-6, subdt=5e-7,
                       opts=port.default_opts(atol=1e-15, rtol=1e-5))
    for k in ("T", "Y", "rho", "c", "subdt"):
        assert np.array_equal(o[k], r[k]), k
    assert o["status"][0] == 1 and r["status"][0] == 1


@pytest.mark.parametrize("name", ["small", "large", "ext", "fitted"])
def test_point_implicit_oracle_vs_reference_golden(name, request):
    """Ri and the diagonal source Jacobian of calculateSourceTermsImp."""
    from oracle import srcimp_oracle
    mk = request.getfixturevalue(name)
    g = _load(name)
    o = srcimp_oracle.srcimp(mk["tables"], g["prop_T"], g["prop_p"], g["prop_rho"], g["prop_Y"])
    assert np.array_equal(o["Ri"], g["srcimp_Ri"])
    ref = g["srcimp_diag"]
    scale = np.abs(ref).max(axis=0, keepdims=True)
    assert (np.abs(o["diag"] - ref) / scale).max() < 1e-14


@pytest.mark.parametrize("name", ["small", "large", "ext", "fitted"])
def test_temperature_from_enthalpy_oracle_vs_reference_golden(name, request):
    """thermoList::THa_p: Newton on the mixture enthalpy with the reference's
    tolerance, iteration cap and [TLow, THigh] clamp."""
    from oracle import props_oracle
    mk = request.getfixturevalue(name)
    g = _load(name)
    T, flag = props_oracle.temperature_from_ha(mk["tables"], g["tha_ha"], g["prop_p"], g["prop_Y"],
                                               g["tha_T0"])
    assert np.array_equal(flag, g["tha_flag"])
    assert np.abs(T - g["tha_T"]).max() < 1e-9
    assert flag[0] == 1   # started at 20 K, below TLow: clamped, then converged inside


@pytest.mark.parametrize("name", ["small", "ext"])
def test_constant_volume_oracle_vs_reference_golden(name, request):
    """chemistrySource with chemSolvers type constVolume: density held, the
    temperature equation on internal energy and cv, the pressure following
    the state (chemistrySource.cpp:885-906, 1022-1055, 1317-1323)."""
    from oracle import port
    mk = request.getfixturevalue(name)
    g = np.load(os.path.join(HERE, "golden", "cv_ref.npz"))
    assert _sha(mk["files"]) == str(g[f"{name}_sha"])
    t = mk["tables"]
    o = port.integrate(port.MechDesc(t), g[f"{name}_in_T"], g[f"{name}_in_p"],
                       g[f"{name}_in_rho"], g[f"{name}_in_Y"], float(g[f"{name}_dt"]),
                       opts=port.default_opts(atol=1e-15, reactor=1))
    for k in ("T", "Y", "c", "subdt", "rho"):
        assert np.array_equal(o[k], g[f"{name}_out_" + k]), k
    assert np.array_equal(o["rho"], g[f"{name}_in_rho"])
    from openhurricane_b200 import mechanism
    mw = 1.0 / np.maximum((o["Y"] / t.W[:, None]).sum(axis=0), 1e-300)
    assert np.array_equal(o["rho"] * (mechanism.RU / mw) * o["T"], g[f"{name}_out_p"])


@pytest.mark.parametrize("name", ["small", "ext"])
def test_temperature_from_energy_oracle_vs_reference_golden(name, request):
    """thermoList::TEa_rho: Newton on the mixture's internal energy at fixed
    density with the reference's tolerance, cap and clamp."""
    from oracle import props_oracle
    mk = request.getfixturevalue(name)
    g = np.load(os.path.join(HERE, "golden", "cv_ref.npz"))
    T, flag = props_oracle.temperature_from_ea(mk["tables"], g[f"{name}_tea_ea"],
                                               g[f"{name}_tea_rho"], g[f"{name}_tea_Y"],
                                               g[f"{name}_tea_T0"])
    assert np.array_equal(flag, g[f"{name}_tea_flag"])
    assert np.abs(T - g[f"{name}_tea_T"]).max() < 1e-9
