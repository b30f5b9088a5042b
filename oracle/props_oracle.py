"""Numpy restatement of the reference's mixture-property path.

TEST INFRASTRUCTURE: the checker of the property kernel, pinned against the
reference's own outputs in tests/golden/*_ref.npz.

  h_i, cp_i   thermo/src/JANAF.cpp:155-199 (mass basis, cp with T clamped,
              h linearly extrapolated outside [TLow, THigh])
  cp          thermoList.cpp:165-190: sum_i cp_i Y_i
  x_i         species/src/speciesList.cpp:208-224 (Yi2Xi)
  mu_i        transport/src/kineticTheory.cpp:37-43, kineticTheory.inl:32-34
  kappa_i     kineticTheory.cpp:51-57: mu_i R_i (cp_i/R_i + 1.25)
  mu, kappa   transport/src/transportList.cpp:238-284 (Wilke)
  D_i         kineticTheory.cpp:118-163 with T^1.5 = T sqrt(T)
"""
import numpy as np

PATM = 1.01325e5
RU = (1.380649e-23 * 6.02214076e23) * 1e3


def properties(t, T, p, Y):
    nsp = t.nsp
    T = np.asarray(T, float)
    p = np.asarray(p, float)
    Y = np.asarray(Y, float)
    W = t.W
    tl, tc, th = t.Trange[:, 0][:, None], t.Trange[:, 1][:, None], t.Trange[:, 2][:, None]
    Tb = T[None, :]
    a = np.where((Tb < tc)[..., None], t.nasa[:, 0, None, :], t.nasa[:, 1, None, :])
    T0 = np.clip(Tb, tl, th)
    cp = ((((a[..., 4] * T0 + a[..., 3]) * T0 + a[..., 2]) * T0 + a[..., 1]) * T0 + a[..., 0])
    h = ((((a[..., 4] / 5.0 * T0 + a[..., 3] / 4.0) * T0 + a[..., 2] / 3.0) * T0
          + a[..., 1] / 2.0) * T0 + a[..., 0]) * T0 + a[..., 5]
    h = h + np.where((Tb < tl) | (Tb > th), cp * (Tb - T0), 0.0)
    cpm = (cp * Y).sum(axis=0)
    Wmean = 1.0 / np.maximum((Y / W[:, None]).sum(axis=0), 1e-300)
    x = np.clip(Y * Wmean[None, :] / W[:, None], 0.0, 1.0)
    xt = x.sum(axis=0)
    x = np.where(xt[None, :] != 1.0, x / xt[None, :], x)
    Tstar = Tb * (1.0 / t.eps_k[:, None])
    om = 1.147 * np.exp(-0.145 * np.log(Tstar)) + 1.0 / (Tstar + 0.5) ** 2
    mu_i = 2.6693e-6 * np.sqrt(W[:, None] * Tb) / ((t.sigma ** 2)[:, None] * om)
    Ri = RU / W[:, None]
    kap_i = mu_i * Ri * (cp / Ri + 1.25)
    phiP = (1.0 / np.sqrt(8.0)) / np.sqrt(1.0 + W[:, None] / W[None, :])
    wiwj = np.sqrt(W[:, None] / W[None, :])
    # phi_i = sum_j phiP(i,j) x_j (1 + sqrt(mu_i/mu_j wiwj(j,i)))^2
    tmp = 1.0 + np.sqrt(mu_i[:, None, :] / mu_i[None, :, :] * wiwj.T[:, :, None])
    phi = (phiP[:, :, None] * x[None, :, :] * tmp ** 2).sum(axis=1)
    mum = (mu_i * x / phi).sum(axis=0)
    kappam = (kap_i * x / phi).sum(axis=0)
    sij = 0.5 * (t.sigma[:, None] + t.sigma[None, :])
    Dc = 1.858e-7 * np.sqrt(1.0 / W[:, None] + 1.0 / W[None, :]) / sij ** 2 * PATM
    r = 1.0 / np.sqrt(t.eps_k[:, None] * t.eps_k[None, :])
    Ts = Tb[None, :, :] * r[:, :, None]
    OmD = np.exp(-0.145 * np.log(Ts)) + 1.0 / (Ts + 0.5) ** 2
    Dij = (Tb * np.sqrt(Tb))[None] * Dc[:, :, None] / (p[None, None, :] * OmD)
    off = ~np.eye(nsp, dtype=bool)
    s = (np.where(off[:, :, None], x[None, :, :] / Dij, 0.0)).sum(axis=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        D = np.where(x < 1.0 - 1e-300, (1.0 - x) / s, 0.0)
    D = np.where(np.isinf(D), 0.0, D)
    return {"ha": h, "cp": cpm, "mu": mum, "kappa": kappam, "D": D}


def species_cp_h(t, T):
    """Mass-basis cp_i and h_i [nsp, n] at temperatures T (JANAF.cpp:155-199)."""
    T = np.asarray(T, float)
    tl, tc, th = t.Trange[:, 0][:, None], t.Trange[:, 1][:, None], t.Trange[:, 2][:, None]
    Tb = T[None, :]
    a = np.where((Tb < tc)[..., None], t.nasa[:, 0, None, :], t.nasa[:, 1, None, :])
    T0 = np.clip(Tb, tl, th)
    cp = ((((a[..., 4] * T0 + a[..., 3]) * T0 + a[..., 2]) * T0 + a[..., 1]) * T0 + a[..., 0])
    h = ((((a[..., 4] / 5.0 * T0 + a[..., 3] / 4.0) * T0 + a[..., 2] / 3.0) * T0
          + a[..., 1] / 2.0) * T0 + a[..., 0]) * T0 + a[..., 5]
    h = h + np.where((Tb < tl) | (Tb > th), cp * (Tb - T0), 0.0)
    return cp, h


def temperature_from_ha(t, ha, p, Y, T0, TLow=50.0, THigh=5000.0, tol=1e-4, max_iter=100):
    """thermoList::THa_p (thermoList.cpp:501-533): Newton on the mixture's
    mass enthalpy, T <- limit(T - (h(T) - ha) / cp(T)), until |dT| <= T0 tol
    or more than max_iter iterations; limit clamps to [TLow, THigh] and sets
    iFlag 0 (below), 1 (inside), 2 (above) (thermoList.cpp:152-163).
    Cell by cell, in the reference's order of operations."""
    ha = np.asarray(ha, float)
    Y = np.asarray(Y, float)
    T0 = np.asarray(T0, float)
    n = ha.shape[0]
    Tout = np.empty(n)
    flag = np.empty(n, np.int32)
    for k in range(n):
        Tnew = T0[k]
        Ttol = T0[k] * tol
        it = 0
        f = 1
        while True:
            Test = Tnew
            cp, h = species_cp_h(t, np.array([Test]))
            hm = float((h[:, 0] * Y[:, k]).sum())
            cpm = float((cp[:, 0] * Y[:, k]).sum())
            v = Test - (hm - ha[k]) / cpm
            if v < TLow:
                f, Tnew = 0, TLow
            elif v > THigh:
                f, Tnew = 2, THigh
            else:
                f, Tnew = 1, v
            it += 1
            if it - 1 > max_iter:
                break
            if not (abs(Tnew - Test) > Ttol):
                break
        Tout[k] = Tnew
        flag[k] = f
    return Tout, flag


def temperature_from_ea(t, ea, rho, Y, T0, TLow=50.0, THigh=5000.0, tol=1e-4, max_iter=100):
    """thermoList::TEa_rho (thermoList.inl:343-348 through thermoList.cpp:501-533):
    the same Newton iteration as THa_p on the mixture's internal energy at
    fixed density, e(T) = sum_i Y_i h_i(T) - p / rho with p = rho Rm T
    (thermoList.inl:302-306, perfectGas.cpp:49-53) and de/dT = cv =
    sum_i Y_i cp_i(T) - Rm (thermoList.inl:145-162)."""
    ea = np.asarray(ea, float)
    rho = np.asarray(rho, float)
    Y = np.asarray(Y, float)
    T0 = np.asarray(T0, float)
    n = ea.shape[0]
    Tout = np.empty(n)
    flag = np.empty(n, np.int32)
    for k in range(n):
        w = 0.0
        for i in range(t.nsp):
            w += Y[i, k] / t.W[i]
        Rm = RU / (1.0 / max(w, 1e-300))
        Tnew = T0[k]
        Ttol = T0[k] * tol
        it = 0
        f = 1
        while True:
            Test = Tnew
            cp, h = species_cp_h(t, np.array([Test]))
            em = float((h[:, 0] * Y[:, k]).sum()) - (rho[k] * Rm * Test) / rho[k]
            cvm = float((cp[:, 0] * Y[:, k]).sum()) - Rm
            v = Test - (em - ea[k]) / cvm
            if v < TLow:
                f, Tnew = 0, TLow
            elif v > THigh:
                f, Tnew = 2, THigh
            else:
                f, Tnew = 1, v
            it += 1
            if it - 1 > max_iter:
                break
            if not (abs(Tnew - Test) > Ttol):
                break
        Tout[k] = Tnew
        flag[k] = f
    return Tout, flag


def mixture_ea(t, T, rho, Y):
    """The mixture's internal energy e = sum_i Y_i h_i - rho Rm T / rho [J/kg]."""
    T = np.asarray(T, float)
    rho = np.asarray(rho, float)
    Y = np.asarray(Y, float)
    cp, h = species_cp_h(t, T)
    w = (Y / t.W[:, None]).sum(axis=0)
    Rm = RU / (1.0 / np.maximum(w, 1e-300))
    return (h * Y).sum(axis=0) - (rho * Rm * T) / rho
