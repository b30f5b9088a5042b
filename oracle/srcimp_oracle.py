"""CPU restatement of the point-implicit source terms
(chemistrySource::calculateSourceTermsImp with withoutLastSpec = true,
chemistrySource.cpp:1412-1450, through omegaCoupled, :422-480).

TEST INFRASTRUCTURE: imported only by tests/, as the checker.

From the analytic Jacobian of the constant-pressure reactor (the oracle's
DyDt / jacobian, bit-exact with the reference's):
  Ri_i     = omega_i W_i
  diag_j   = J_jj - (W_j / W_L) J_jL + J_jT W_j (e_L - e_j) / (rho c_v),   j < nsp - 1
with L the last species (its concentration follows from the others at fixed
density: dc_L/dc_j = -W_j / W_L, reactionTypes.cpp:761-790, :793-832),
e_i = h_i - R_i T the species' mass internal energy (thermo.inl:168-171) and
c_v = c_p - R_mix the mixture's (thermoList.inl:145-149).
"""
from __future__ import annotations

import numpy as np

from . import port, props_oracle


def srcimp(t, T, p, rho, Y):
    T = np.asarray(T, np.float64)
    rho = np.asarray(rho, np.float64)
    Y = np.asarray(Y, np.float64)
    nsp = t.nsp
    c = rho[None, :] * Y / t.W[:, None]
    f, J = port.rhs_jac(port.MechDesc(t), c, T, p)
    Ri = f[:, :nsp].T * t.W[:, None]
    pr = props_oracle.properties(t, T, p, Y)
    R = props_oracle.RU / t.W
    e = pr["ha"] - R[:, None] * T[None, :]
    Rmix = props_oracle.RU * (Y / t.W[:, None]).sum(axis=0)
    cv = pr["cp"] - Rmix
    L = nsp - 1
    diag = np.empty((nsp - 1, T.shape[0]))
    for j in range(nsp - 1):
        diag[j] = (J[:, j, j] - (t.W[j] / t.W[L]) * J[:, j, L]
                   + J[:, j, nsp] * t.W[j] * (e[L] - e[j]) / (rho * cv))
    return {"Ri": Ri, "diag": diag}
