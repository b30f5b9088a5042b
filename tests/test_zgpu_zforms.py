"""GPU parity of the reactor and rate forms beyond the plain path: the
extended rate forms (SRI, HIGH, REV, FORD / RORD, PLOG, LT, units), the
fitted ones (JAN, FIT1, RLT, COLLEFF), the constant-volume reactor and
temperature from internal energy, against the oracle and the reference's
golden outputs. Collected after the plain-path GPU tests (test_zgpu_parity.py),
whose helpers and tolerances these share."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import test_zgpu_parity as P  # noqa: E402  (helpers and tolerances)
from test_zgpu_parity import (PARITY, T_RTOL, Y_FLOOR, Y_RTOL, _assert_close,  # noqa: E402
                              _cells, _cuda, _gpu_integrate, _mech, _oracle)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["ext", "fitted"])
def test_extended_forms_against_reference_golden_outputs(name, request):
    P.test_against_reference_golden_outputs(name, request)


@pytest.mark.parametrize("name", ["ext", "fitted"])
def test_extended_forms_rhs_jacobian_vs_reference_golden(name, request):
    P.test_rhs_jacobian_vs_reference_golden(name, request)


@pytest.mark.parametrize("name", ["ext", "fitted"])
def test_extended_forms_point_implicit_source_terms_vs_reference_golden(name, request):
    P.test_point_implicit_source_terms_vs_reference_golden(name, request)


@pytest.mark.parametrize("kernel", [0, 2])
def test_extended_rate_forms_parity_vs_oracle(ext, kernel):
    """SRI fall-off, explicit reverse parameters (REV) on Arrhenius and
    third-body reactions, FORD / RORD orders and unit keywords, through the
    cell-group kernels, against the oracle (pinned to the reference on this
    mechanism), over a flow step of 1e-7 s: over 1e-6 s some of this
    mechanism's cells answer one-ulp changes of their inputs with 1e-6
    changes of T in the oracle itself (every seed tried), which no parity
    tolerance between two libms survives; over 1e-7 s the largest such change
    on these cells is 1.6e-10. They take at most 37083 Newton iterations each
    in the oracle; the GPU run carries a cap of 1000000 per cell so that a
    cell taking another path ends the test with a failure instead of running
    on."""
    t = ext["tables"]
    assert (t.rate_type == 5).sum() == 2 and (t.reversible == 2).sum() == 3
    assert (t.rate_type == 6).sum() == 3 and (t.rate_type == 7).sum() == 1
    assert t.activated.sum() == 1
    T, p, rho, Y = _cells(t, 128, seed=13)
    m = _mech(t)
    m.set_tuning(kernel, 64)
    g = _gpu_integrate(m, T, p, rho, Y, 1e-7, max_newton_total=1000000, **PARITY)
    o = _oracle(t, T, p, rho, Y, 1e-7, key="ext128", **PARITY)
    assert np.array_equal(g["status"] & 12, np.zeros_like(g["status"]))
    _assert_close(g, o, f"extended forms, kernel {kernel}")
    c0 = rho[None, :] * Y / t.W[:, None]
    Ri_o = (o["c"] - c0) / 1e-7 * t.W[:, None]
    scale = np.abs(Ri_o).max(axis=0, keepdims=True) + 1e-300
    assert (np.abs(g["Ri"] - Ri_o) / scale).max() < 1e-5


@pytest.mark.parametrize("name,seed,dt", [("small", 17, 1e-7), ("ext", 19, 3e-8)])
@pytest.mark.parametrize("kernel", [0, 2])
def test_constant_volume_reactor_parity_vs_oracle(name, seed, dt, kernel, request):
    """chemSolvers type constVolume: density held, the temperature equation on
    internal energy and cv, p following the state (for PLOG rates), through
    the cell-group kernel, against the oracle (pinned to the reference). The
    step lengths keep these cells well conditioned (one-ulp input changes move
    T by at most 2e-11 in the oracle) and cheap (at most 44515 Newton
    iterations a cell); the cap bounds a cell that would take another path."""
    mk = request.getfixturevalue(name)
    t = mk["tables"]
    T, p, rho, Y = _cells(t, 96, seed=seed)
    m = _mech(t)
    m.set_tuning(kernel, 64)
    g = _gpu_integrate(m, T, p, rho, Y, dt, reactor=1, max_newton_total=1000000, **PARITY)
    o = _oracle(t, T, p, rho, Y, dt, key=f"cv-{name}", reactor=1, **PARITY)
    assert np.array_equal(g["status"] & 12, np.zeros_like(g["status"]))
    _assert_close(g, o, f"constant volume {name}, kernel {kernel}")
    assert np.array_equal(g["rho"], rho)
    assert (g["T"] > T).any()


@pytest.mark.parametrize("name", ["small", "ext"])
def test_constant_volume_reactor_vs_reference_golden(name, request):
    """The reference's own constant-volume outputs at its default rtol:
    statistical agreement as for the constant-pressure golden cases."""
    import os
    mk = request.getfixturevalue(name)
    here = os.path.dirname(os.path.abspath(__file__))
    g0 = np.load(os.path.join(here, "golden", "cv_ref.npz"))
    m = _mech(mk["tables"])
    g = _gpu_integrate(m, g0[name + "_in_T"], g0[name + "_in_p"], g0[name + "_in_rho"],
                       g0[name + "_in_Y"], float(g0[name + "_dt"]), atol=1e-15, reactor=1,
                       max_newton_total=1000000)
    ref_T, ref_Y = g0[name + "_out_T"], g0[name + "_out_Y"]
    dT = np.abs(g["T"] - ref_T) / ref_T
    assert dT.max() < 1e-4
    dY = np.abs(g["Y"] - ref_Y) - Y_RTOL * np.abs(ref_Y) - Y_FLOOR
    ok = (dT <= T_RTOL) & (dY.max(axis=0) <= 0.0)
    assert ok.mean() >= 0.9, f"{ok.mean():.3f} of cells within parity tolerance"
    assert np.array_equal(g["rho"], g0[name + "_in_rho"])


@pytest.mark.parametrize("kernel", [1, 3, 4])
def test_constant_volume_refused_by_thread_per_cell_kernels(small, kernel):
    from openhurricane_b200 import _capi
    t = small["tables"]
    T, p, rho, Y = _cells(t, 8, seed=18)
    m = _mech(t)
    m.set_tuning(kernel, 64)
    with pytest.raises(_capi.HcError, match="constant-pressure"):
        _gpu_integrate(m, T, p, rho, Y, 1e-7, reactor=1, **PARITY)


@pytest.mark.parametrize("kernel", [1, 3, 4])
def test_extended_rate_forms_refused_by_thread_per_cell_kernels(ext, kernel):
    from openhurricane_b200 import _capi
    t = ext["tables"]
    T, p, rho, Y = _cells(t, 8, seed=14)
    m = _mech(t)
    m.set_tuning(kernel, 64)
    with pytest.raises(_capi.HcError, match="SRI"):
        _gpu_integrate(m, T, p, rho, Y, 1e-6, **PARITY)


def test_extended_rate_forms_source_terms_vs_oracle(ext):
    from oracle import port
    dev = _cuda()
    t = ext["tables"]
    T, p, rho, Y = _cells(t, 256, seed=15)
    m = _mech(t)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    Ri = m.source_terms(d(T), d(p), d(rho), d(Y)).cpu().numpy()
    c = rho[None, :] * Y / t.W[:, None]
    f, _ = port.rhs_jac(port.MechDesc(t), c, T, p)
    ref = f[:, : t.nsp].T * t.W[:, None]
    sc = np.abs(ref).max(axis=0, keepdims=True) + 1e-300
    assert (np.abs(Ri - ref) / sc).max() < 1e-11


@pytest.mark.parametrize("name", ["small", "ext"])
def test_temperature_from_energy_vs_reference_golden(name, request):
    """hc_temperature_from_energy against thermoList::TEa_rho's own outputs."""
    import os
    mk = request.getfixturevalue(name)
    here = os.path.dirname(os.path.abspath(__file__))
    g0 = np.load(os.path.join(here, "golden", "cv_ref.npz"))
    dev = _cuda()
    m = _mech(mk["tables"])
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    T, flag = m.temperature_from_energy(d(g0[name + "_tea_ea"]), d(g0[name + "_tea_Y"]),
                                        d(g0[name + "_tea_rho"]), d(g0[name + "_tea_T0"]))
    assert np.array_equal(flag.cpu().numpy(), g0[name + "_tea_flag"])
    assert np.abs(T.cpu().numpy() - g0[name + "_tea_T"]).max() < 1e-6


@pytest.mark.parametrize("kernel", [0, 2])
def test_fitted_rates_parity_vs_oracle(fitted, kernel):
    """Janev (JAN), power-series (FIT1), reverse Landau-Teller (RLT) and
    collision-efficiency (COLLEFF) rates through the cell-group kernel against
    the oracle (pinned to the reference); over 1e-7 s these cells are well
    conditioned (one-ulp input changes move T by 2.5e-9 relative in the
    oracle) and take at most 39150 Newton iterations each."""
    t = fitted["tables"]
    T, p, rho, Y = _cells(t, 96, seed=23)
    m = _mech(t)
    m.set_tuning(kernel, 64)
    g = _gpu_integrate(m, T, p, rho, Y, 1e-7, max_newton_total=1000000, **PARITY)
    o = _oracle(t, T, p, rho, Y, 1e-7, key="fitted96", **PARITY)
    assert np.array_equal(g["status"] & 12, np.zeros_like(g["status"]))
    _assert_close(g, o, f"fitted rates, kernel {kernel}")


@pytest.mark.parametrize("collision_b", [0.0, 0.5])
def test_fitted_rates_rhs_jacobian_vs_oracle(fitted, collision_b, tmp_path):
    """DyDt and the Jacobian of the fitted-rates mechanism; with b = 0.5 on the
    collision reaction its dk/dT (the reference's Arrhenius derivative at k
    times dZ/dT) is non-zero."""
    from oracle import port
    from openhurricane_b200 import mechanism, synth
    dev = _cuda()
    t = fitted["tables"]
    if collision_b:
        t = mechanism.compile_mechanism(*synth.write_chemkin(
            synth.fitted_rates_mechanism(collision=(1e-22, collision_b, 0.0)), str(tmp_path)))
    rng = np.random.default_rng(3)
    n = 16
    T = rng.uniform(800.0, 3000.0, n)
    p = rng.uniform(1.0, 5.0, n) * 101325.0
    c = rng.dirichlet(np.full(t.nsp, 0.5), n).T.copy() * 0.01
    m = _mech(t)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dydt, J = m.rhs_jacobian(d(c), d(T), d(p))
    ref_f, ref_J = port.rhs_jac(port.MechDesc(t), c, T, p)
    sf = np.abs(ref_f).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(dydt.cpu().numpy() - ref_f) / sf).max() < 1e-11
    sJ = np.abs(ref_J).max(axis=(1, 2), keepdims=True) + 1e-300
    assert (np.abs(J.cpu().numpy() - ref_J) / sJ).max() < 1e-11
