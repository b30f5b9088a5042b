"""The device rate-law helpers (openhurricane_b200/csrc/rtc_base.cuh), compiled
for the host with g++, against the reference's formulas restated here:
the SRI fall-off function (reactionRateTypes/src/fallOffFunctions.cpp:54-79,
SRI::F, SRI::DFDci, SRI::DFDT; the device path folds 1/Pr * dPr/dci out of
DFDci, as it forms the rank-one third-body column once per reaction, and the
check multiplies it back in) and the PLOG table (logInterpolationRR.cpp:78-147
k, :149-226 DkDT, restated loop for loop; the device form evaluates only the
interval the reference's loop ends on) and the Landau-Teller rate
(LandauTellerRR.cpp:37-99)."""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TINY = 1e-15


def _ref(a, b, c, d, e, T, Pr, F, DPrDT, DPrDci):
    base = a * math.exp(-b / T) + math.exp(-T / c)
    logPr = math.log10(max(Pr, TINY))
    X = 1.0 / (1.0 + logPr * logPr)
    Fv = d * math.pow(base, X) * math.pow(T, e)
    dXdc = -X * X * 2.0 * math.log10(Pr) / Pr / math.log(10.0) * DPrDci
    dFdci = F * dXdc * math.log(base)
    dXdPr = -X * X * 2.0 * math.log10(Pr) / Pr / math.log(10.0)
    dFdT = F * (e / T + dXdPr * DPrDT * math.log(base) +
                X * (a * b * math.exp(-b / T) / (T * T) - math.exp(-T / c) / c) / base)
    return Fv, dFdT, dFdci


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("helpers") / "rate_helpers")
    inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    subprocess.check_call([gxx, "-O2", "-std=c++17", "-I", inc, "-o", out,
                           os.path.join(HERE, "cpp", "rate_helpers.cpp")])
    return out


def test_sri_helpers_match_the_reference_formulas(exe):
    rng = np.random.default_rng(7)
    rows = []
    for _ in range(200):
        a, b, c = rng.uniform(0.3, 3.0), rng.uniform(50.0, 1500.0), rng.uniform(200.0, 3000.0)
        d, e = (1.0, 0.0) if rng.uniform() < 0.5 else (rng.uniform(0.7, 1.3), rng.uniform(-0.5, 0.5))
        T = rng.uniform(300.0, 3000.0)
        Pr = 10.0 ** rng.uniform(-6.0, 6.0)
        F = rng.uniform(0.1, 2.0)
        rows.append((a, b, c, d, e, T, Pr, F, rng.uniform(-1e-2, 1e-2) * Pr))
    txt = "\n".join("S " + " ".join(repr(float(v)) for v in r) for r in rows) + "\n"
    out = subprocess.run([exe], input=txt, capture_output=True, text=True, check=True).stdout
    got = np.array([[float(x) for x in l.split()] for l in out.strip().splitlines()])
    assert got.shape == (len(rows), 3)
    for r, g in zip(rows, got):
        DPrDci = 0.37 * r[6]
        Fv, dFdT, dFdci = _ref(*r, DPrDci)
        assert abs(g[0] - Fv) <= 1e-14 * abs(Fv)
        assert abs(g[1] - dFdT) <= 1e-12 * max(abs(dFdT), 1e-300)
        fold = g[2] * (1.0 / r[6]) * DPrDci
        assert abs(fold - dFdci) <= 1e-12 * max(abs(dFdci), 1e-300)


def _arr(a, T):
    """ArrheniusRR::k (ArrheniusRR.cpp:37-47) and ::DkDT (ArrheniusRR.hpp:96-99)."""
    k = a[0]
    if abs(a[1]) > 1e-300:
        k *= math.pow(T, a[1])
    if abs(a[2]) > 1e-300:
        k *= math.exp(-a[2] / T)
    return k


def _arr_dkdt(a, kj, T):
    invT = 1.0 / max(T, TINY)
    return kj * invT * (a[1] + a[2] * invT)


def _plog_ref(pp, ka, p, T):
    """logInterpolationRR::k and ::DkDT, loop for loop."""
    n = len(pp)
    if p <= pp[0]:
        k = _arr(ka[0], T)
        d = _arr_dkdt(ka[0], k, T)
        for i in range(n - 1):
            if pp[i + 1] > pp[i]:
                break
            ki = _arr(ka[i + 1], T)
            k += ki
            d += _arr_dkdt(ka[i + 1], ki, T)
        return k, d
    if p >= pp[-1]:
        k = _arr(ka[-1], T)
        return k, _arr_dkdt(ka[-1], k, T)
    k = d = None
    for i in range(n - 1):
        if p < pp[i + 1]:
            k0 = _arr(ka[i], T)
            dk0 = _arr_dkdt(ka[i], k0, T)
            for j in range(i - 1, -1, -1):
                if pp[j + 1] > pp[j]:
                    break
                kj = _arr(ka[j], T)
                k0 += kj
                dk0 += _arr_dkdt(ka[j], kj, T)
            k1 = _arr(ka[i + 1], T)
            dk1 = _arr_dkdt(ka[i + 1], k1, T)
            for j in range(i + 1, n - 1):
                if pp[j + 1] > pp[j]:
                    break
                kj = _arr(ka[j + 1], T)
                k1 += kj
                dk1 += _arr_dkdt(ka[j + 1], kj, T)
            lnp0, lnp1, lnp = math.log(pp[i]), math.log(pp[i + 1]), math.log(p)
            lnk0, lnk1 = math.log(k0), math.log(k1)
            lnk = lnk0 + (lnk1 - lnk0) * (lnp - lnp0) / (lnp1 - lnp0)
            k = math.exp(lnk) if lnk < 709.0 else math.inf   # exp overflows to inf in C
            d = 1.0 / k0 * dk0 + (1.0 / k1 * dk1 - 1.0 / k0 * dk0) * (lnp - lnp0) / (lnp1 - lnp0)
    return k, k * d


def test_plog_helpers_match_the_reference_loops(exe):
    rng = np.random.default_rng(8)
    cases = []
    for _ in range(300):
        n = int(rng.integers(1, 6))
        pp = sorted(float(x) for x in 10.0 ** rng.uniform(3.0, 7.0, n))
        if n >= 3 and rng.uniform() < 0.5:
            pp[1] = pp[0]            # a repeated lower pressure (rates add)
        if n >= 2 and pp[-1] == pp[-2]:
            pp[-1] *= 2.0
        ka = [(float(10.0 ** rng.uniform(6.0, 14.0)), float(rng.uniform(-1.0, 2.0)),
               float(rng.uniform(0.0, 3e4))) for _ in range(n)]
        p = float(10.0 ** rng.uniform(2.5, 7.5))
        T = float(rng.uniform(300.0, 3000.0))
        cases.append((pp, ka, p, T))
    txt = "".join(f"P {len(pp)} {p!r} {T!r} " + " ".join(
        f"{q!r} {a[0]!r} {a[1]!r} {a[2]!r}" for q, a in zip(pp, ka)) + "\n"
        for pp, ka, p, T in cases)
    out = subprocess.run([exe], input=txt, capture_output=True, text=True, check=True).stdout
    got = np.array([[float(x) for x in l.split()] for l in out.strip().splitlines()])
    assert got.shape == (len(cases), 2)
    for (pp, ka, p, T), g in zip(cases, got):
        k, d = _plog_ref(pp, ka, p, T)
        if not math.isfinite(k):
            # far outside the two highest pressures the extrapolation overflows
            assert g[0] == math.inf
            continue
        assert abs(g[0] - k) <= 1e-12 * abs(k), (pp, p, T)
        assert abs(g[1] - d) <= 1e-11 * max(abs(d), 1e-300) + 1e-12 * abs(k) / T, (pp, p, T)


def test_plog_oracle_matches_the_reference_loops(ext):
    """The oracle's PLOG rates (chem_oracle.c) against the same restatement,
    on the extended mechanism's three tables at pressures below, inside and
    above each."""
    from oracle import port
    t = ext["tables"]
    md = port.MechDesc(t)
    rows = np.flatnonzero(t.rate_type == 6)
    assert len(rows) == 3
    c = np.full(t.nsp, 1e-3)
    for p in (1e3, 2e4, 1.5e5, 4e5, 3e6, 5e7):
        for T in (700.0, 1500.0, 2600.0):
            kf = port.rates(md, T, c, p)[:, 0]
            for r in rows:
                b, e = t.plog_ptr[r], t.plog_ptr[r + 1]
                k, _ = _plog_ref([float(x) for x in t.plog_p[b:e]],
                                 [tuple(float(v) for v in a) for a in t.plog_arr[b:e]], p, T)
                assert kf[r] == k


def _lt_ref(A, b, Ta, B, C, T):
    """LandauTellerRR::k and ::DkDT as written."""
    lta = A
    if abs(b) > 1e-300:
        lta *= math.pow(T, b)
    e = 0.0
    if abs(Ta) > 1e-300:
        e -= Ta / T
    if abs(B) > 1e-300:
        e += B / math.pow(T, 1.0 / 3.0)
    if abs(C) > 1e-300:
        e += C / math.pow(T, 2.0 / 3.0)
    k = lta * math.exp(e) if abs(e) > 1e-300 else lta
    lta = A * (math.pow(T, b) if abs(b) > 1e-300 else 1.0)
    ea, d = 0.0, 0.0
    if abs(Ta) > 1e-300:
        ea -= Ta / T
        d += Ta / T
    if abs(B) > 1e-300:
        bt = B / np.cbrt(T)
        ea += bt
        d -= bt / 3
    if abs(C) > 1e-300:
        ct = C / math.pow(T, 2.0 / 3.0)
        ea += ct
        d -= 2 * ct / 3
    if abs(ea) > 1e-300:
        lta *= math.exp(ea)
    return k, lta * (b + d) / T


def test_landau_teller_helpers_match_the_reference(exe):
    rng = np.random.default_rng(9)
    cases = [(float(10.0 ** rng.uniform(6, 14)), float(rng.uniform(-1, 2)),
              float(rng.uniform(0, 3e4)), float(rng.uniform(-40, 40)), float(rng.uniform(-90, 90)),
              float(rng.uniform(300, 3000))) for _ in range(200)]
    cases.append((1e10, 0.0, 0.0, 0.0, 0.0, 1000.0))
    txt = "".join("L " + " ".join(repr(v) for v in c) + "\n" for c in cases)
    out = subprocess.run([exe], input=txt, capture_output=True, text=True, check=True).stdout
    got = np.array([[float(x) for x in l.split()] for l in out.strip().splitlines()])
    for c, g in zip(cases, got):
        k, d = _lt_ref(*c)
        assert abs(g[0] - k) <= 1e-13 * abs(k), c
        assert abs(g[1] - d) <= 1e-12 * max(abs(d), 1e-300) + 1e-14 * abs(k) / c[-1], c


def test_janev_and_power_series_helpers_match_the_reference(exe):
    """JanevRR (JanevRR.cpp:37-88) and powerSeriesRR (powerSeriesRateRR.cpp:37-74)."""
    rng = np.random.default_rng(10)
    jan, fit = [], []
    for _ in range(100):
        A, b, Ta = float(10.0 ** rng.uniform(6, 14)), float(rng.uniform(-1, 2)), float(rng.uniform(0, 3e4))
        bn = [float(rng.uniform(-1, 1) * 0.3 / 8.0 ** n) for n in range(9)]
        T = float(rng.uniform(300, 3000))
        jan.append((A, b, Ta, bn, T))
        fn = [float(rng.uniform(-300, 300)), float(rng.uniform(-1e5, 1e5)),
              float(rng.uniform(-1e7, 1e7)), float(rng.uniform(-1e9, 1e9))]
        fit.append((A, b, fn, T))
    txt = "".join(f"J {A!r} {b!r} {Ta!r} " + " ".join(repr(x) for x in bn) + f" {T!r}\n"
                  for A, b, Ta, bn, T in jan)
    txt += "".join(f"F {A!r} {b!r} " + " ".join(repr(x) for x in fn) + f" {T!r}\n"
                   for A, b, fn, T in fit)
    out = subprocess.run([exe], input=txt, capture_output=True, text=True, check=True).stdout
    got = np.array([[float(x) for x in l.split()] for l in out.strip().splitlines()])
    for (A, b, Ta, bn, T), g in zip(jan, got[:100]):
        lnT = math.log(T)
        e = -Ta / T + sum(bn[n] * math.pow(lnT, n) for n in range(9))
        k = A * math.pow(T, b) * math.exp(e)
        d = bn[1] + sum(n * bn[n] * math.pow(lnT, n - 1) for n in range(2, 9))
        dk = k * (b + Ta / T + d) / T
        assert abs(g[0] - k) <= 1e-13 * abs(k)
        assert abs(g[1] - dk) <= 1e-12 * abs(dk) + 1e-14 * abs(k) / T
    for (A, b, fn, T), g in zip(fit, got[100:]):
        e = sum(fn[n] / math.pow(T, n + 1) for n in range(4))
        k = A * math.pow(T, b) * math.exp(e)
        dk = k * (b - sum((n + 1) * fn[n] / math.pow(T, n + 1) for n in range(4))) / T
        assert abs(g[0] - k) <= 1e-13 * abs(k)
        assert abs(g[1] - dk) <= 1e-12 * abs(dk) + 1e-14 * abs(k) / T


def test_collision_helpers_match_the_reference(exe):
    """collisionRR (collisionRR.hpp:94-107, 146-169): k = min(1, Arrhenius) Zb,
    dk/dT = (k > 1 ? k (b + Ta/T) / T : 0) dZb/dT, on both sides of k = 1 and
    of the efficiency's cap at 1."""
    rng = np.random.default_rng(12)
    cases = []
    for i in range(120):
        A = float(10.0 ** rng.uniform(-34, 2))
        b = float(rng.choice([0.0, rng.uniform(-1, 1)]))
        Ta = float(rng.choice([0.0, rng.uniform(0, 2e4)]))
        x = (float(6.02214076e23 * rng.uniform(2, 6) ** 2), float(rng.uniform(2e3, 5e5)),
             0.0)
        x = (x[0], x[1], x[1] / 4.0)
        cases.append((A, b, Ta, x, float(rng.uniform(300, 3000))))
    txt = "".join(f"K {A!r} {b!r} {Ta!r} {x[0]!r} {x[1]!r} {x[2]!r} {T!r}\n"
                  for A, b, Ta, x, T in cases)
    out = subprocess.run([exe], input=txt, capture_output=True, text=True, check=True).stdout
    got = np.array([[float(v) for v in l.split()] for l in out.strip().splitlines()])
    seen = set()
    for (A, b, Ta, x, T), g in zip(cases, got):
        gam = min(1.0, A * math.pow(T, b) * math.exp(-Ta / T))
        k = gam * (x[0] * math.sqrt(x[1] * T))
        dk = (k * (b + Ta / T) / T if k > 1.0 else 0.0) * (x[0] * math.sqrt(x[2] / T))
        seen.add((gam == 1.0, k > 1.0))
        assert abs(g[0] - k) <= 1e-13 * abs(k)
        assert abs(g[1] - dk) <= 1e-12 * abs(dk) + 1e-300
    assert {(False, True), (False, False), (True, True)} <= seen
