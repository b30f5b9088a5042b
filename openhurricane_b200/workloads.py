"""Seeded synthetic workloads of the chemistry source-term benchmarks.

There is no public dataset for this path; every input is generated here from
a seed with the shapes and distributions of the workloads:

  small       9 species / 21 reactions, T U[1000,2500] K, p U[1,5] atm,
              Y ~ Dirichlet(0.5), dt = 1e-6 s (4096 cells)
  batched     same mechanism, 1,048,576 cells: 20 % near ignition
              (T U[1100,1300] K, Dirichlet(2) over the reactant species H2,
              O2, N2, all other species zero) and 80 % near equilibrium
              (random states relaxed by the FP64 integrator, then jittered),
              dt = 1e-5 s
  large       53 species / 325 reactions, T U[800,2800] K, p U[0.5,10] atm,
              Y ~ Dirichlet(0.3), 262,144 cells

Solver options: the reference's 0-D application configuration
(applications/chemSolvers/chemSolvers.hpp: ImplicitEuler with maxstep 10000,
atol 1e-11, rtol 1e-4) unless stated otherwise.
"""
from __future__ import annotations

import dataclasses
import tempfile
from typing import Dict, Optional

import numpy as np

from . import synth
from .mechanism import MechTables, compile_mechanism

SOLVER_OPTS = dict(atol=1e-11, rtol=1e-4)
REACTANTS_SMALL = ("H2", "O2", "N2")


@dataclasses.dataclass
class Workload:
    name: str
    tables: MechTables
    files: tuple
    T: np.ndarray
    p: np.ndarray
    rho: np.ndarray
    Y: np.ndarray
    dt: float
    note: str = ""

    @property
    def n(self) -> int:
        return int(self.T.shape[0])


def mechanism_files(which: str, out_dir: Optional[str] = None):
    m = synth.small_mechanism() if which == "small" else synth.large_mechanism()
    d = out_dir or tempfile.mkdtemp(prefix=f"hc_{which}_")
    files = synth.write_chemkin(m, d)
    return m, files, compile_mechanism(*files)


def small_cells(n: int, seed: int = 1001):
    return synth.dirichlet_cells(9, n, seed=seed)


def large_cells(n: int, seed: int = 3003):
    return synth.dirichlet_cells(53, n, seed=seed, T_range=(800.0, 2800.0),
                                 p_atm_range=(0.5, 10.0), alpha=0.3)


def make_small(n: int = 4096, seed: int = 1001, out_dir=None) -> Workload:
    _, files, t = mechanism_files("small", out_dir)
    c = small_cells(n, seed)
    return Workload("small", t, files, c.T, c.p, synth.mixture_density(t.W, c), c.Y, 1e-6)


def make_large(n: int = 262144, seed: int = 3003, out_dir=None) -> Workload:
    _, files, t = mechanism_files("large", out_dir)
    c = large_cells(n, seed)
    return Workload("large", t, files, c.T, c.p, synth.mixture_density(t.W, c), c.Y, 1e-6)


def gibbs_rt(t: MechTables, T: np.ndarray) -> np.ndarray:
    """Molar standard Gibbs energy over Ru T of every species, [nsp, n], from
    the NASA-7 polynomials (the mass-basis table divided by R_i)."""
    T = np.asarray(T, np.float64)
    out = np.empty((t.nsp, T.shape[0]))
    for i in range(t.nsp):
        hi = T >= t.Trange[i, 1]
        a = np.where(hi[None, :], t.nasa[i, 1][:, None], t.nasa[i, 0][:, None]) / t.Ri[i]
        h_rt = a[0] + a[1] * T / 2 + a[2] * T ** 2 / 3 + a[3] * T ** 3 / 4 + a[4] * T ** 4 / 5 + a[5] / T
        s_r = a[0] * np.log(T) + a[1] * T + a[2] * T ** 2 / 2 + a[3] * T ** 3 / 3 + a[4] * T ** 4 / 4 + a[6]
        out[i] = h_rt - s_r
    return out


def equilibrium_tp(t: MechTables, T, p, Y, iters: int = 200):
    """Chemical equilibrium mass fractions at fixed T and p with the element
    content of Y (element-potential method, damped Newton on the element
    potentials and ln of the total moles, vectorised over cells). At the
    equilibrium composition every reaction's forward and reverse rates
    balance (Kc is built from the same Gibbs energies), so the state is a
    fixed point of the reactor."""
    T = np.asarray(T, np.float64)
    p = np.asarray(p, np.float64)
    A = t.elem_matrix[np.abs(t.elem_matrix).sum(axis=1) > 0]          # [ne, nsp]
    ne = A.shape[0]
    b = A @ (np.asarray(Y) / t.W[:, None])                             # kmol element / kg
    g = gibbs_rt(t, T) + np.log(p / 101325.0)[None, :]                  # [nsp, n]
    n = T.shape[0]
    pi = np.zeros((ne, n))
    nu = np.log(np.maximum(b.sum(axis=0), 1e-30))
    present = (A.T @ (b > 0)) == A.sum(axis=0)[:, None]                  # species made of present elements
    for _ in range(iters):
        lx = -g + A.T @ pi
        lx = np.where(present, np.minimum(lx, 50.0), -np.inf)
        x = np.exp(lx)
        nmol = np.exp(nu)[None, :] * x
        Fe = A @ nmol - b
        Fx = x.sum(axis=0) - 1.0
        J = np.zeros((n, ne + 1, ne + 1))
        J[:, :ne, :ne] = np.einsum("ei,fi,in->nef", A, A, nmol)
        J[:, :ne, ne] = (A @ nmol).T
        J[:, ne, :ne] = (A @ x).T
        rhs = -np.concatenate([Fe, Fx[None, :]], axis=0).T              # [n, ne+1]
        # elements absent from a cell: keep their potential fixed
        absent = (b <= 0).T
        for e in range(ne):
            J[absent[:, e], e, :] = 0.0
            J[absent[:, e], :, e] = 0.0
            J[absent[:, e], e, e] = 1.0
            rhs[absent[:, e], e] = 0.0
        d = np.linalg.solve(J, rhs[..., None])[..., 0]
        step = np.max(np.abs(d), axis=1)
        lam = np.minimum(1.0, 2.0 / np.maximum(step, 1e-300))
        pi += (lam[:, None] * d[:, :ne]).T
        nu += lam * d[:, ne]
        if np.max(step) < 1e-12:
            break
    lx = np.where(present, -g + A.T @ pi, -np.inf)
    nmol = np.exp(nu)[None, :] * np.exp(lx)
    Yeq = nmol * t.W[:, None]
    return Yeq / Yeq.sum(axis=0, keepdims=True)


def make_batched(n: int = 1048576, seed: int = 2002, frac_ignition: float = 0.2,
                 relax=None, pool: int = 8192, relax_time: float = 1e-4,
                 out_dir=None) -> Workload:
    """20 % ignition cells + 80 % near-equilibrium cells.

    Near-equilibrium cells come from a pool of random states: by default each
    pool state is replaced by its chemical equilibrium at its own T and p
    (equilibrium_tp; pool temperatures U[1500, 2800] K), or, when
    `relax(T, p, rho, Y, dt) -> (T, rho, Y)` is given, by integrating it over
    relax_time. The pool is tiled over the near-equilibrium cells with a
    seeded jitter of +-2 K in T so that no two cells are identical."""
    _, files, t = mechanism_files("small", out_dir)
    rng = np.random.default_rng(seed)
    n_ign = int(round(frac_ignition * n))
    idx = [t.names.index(s) for s in REACTANTS_SMALL]
    ign = synth.ignition_cells(t.nsp, n_ign, seed=seed + 1, reactant_idx=idx)
    base = synth.dirichlet_cells(t.nsp, pool, seed=seed + 2)
    if relax is None:
        Tb = np.random.default_rng(seed + 3).uniform(1500.0, 2800.0, pool)
        Yb = equilibrium_tp(t, Tb, base.p, base.Y)
    else:
        rho_b = synth.mixture_density(t.W, base)
        Tb, rhob, Yb = relax(base.T, base.p, rho_b, base.Y, relax_time)
    n_eq = n - n_ign
    pick = rng.integers(0, pool, n_eq)
    T_eq = Tb[pick] + rng.uniform(-2.0, 2.0, n_eq)
    p_eq = base.p[pick]
    Y_eq = Yb[:, pick]
    T = np.concatenate([ign.T, T_eq])
    p = np.concatenate([ign.p, p_eq])
    Y = np.ascontiguousarray(np.concatenate([ign.Y, Y_eq], axis=1))
    perm = rng.permutation(n)     # interleave the two populations
    T, p, Y = T[perm], p[perm], np.ascontiguousarray(Y[:, perm])
    cells = synth.Cells(T, p, Y)
    rho = synth.mixture_density(t.W, cells)
    return Workload("batched", t, files, T, p, rho, Y, 1e-5,
                    note=f"{n_ign} ignition + {n_eq} near-equilibrium cells")


def flop_model(t: MechTables, transcendental: float = 20.0) -> Dict[str, float]:
    """Algorithmic FLOPs of one right-hand side, one analytic Jacobian, one
    LU factorisation and one LU solve of the n = nsp+1 system.

    Counting convention: add/mul/div = 1, fused multiply-add = 2, each FP64
    exp/log/pow = `transcendental` FLOP. Per reaction the necessary work is
    kf (1 exp of b ln T - Ta/T), Kc (1 exp, ~2 FLOP per species term), the
    concentration products (one pow per non-unit order, 1 mul per species)
    and, for the Jacobian, one product per (reactant, reactant) pair plus
    dq/dT; third-body reactions add 2 FLOP per species (M) and, in the
    Jacobian, 3 FLOP per species column and participant; Troe fall-off adds
    6 transcendentals for F and 12 for its derivatives. Species thermo:
    1 log + ~40 FLOP each. The temperature row is 2 nsp^2 + 10 nsp.
    LU: 2(n^3/3 - n^2/2 + n/6), solve: 2 n^2."""
    nsp = t.nsp
    n = nsp + 1
    tr = transcendental
    f_rhs = nsp * (tr + 40.0)
    f_jac = f_rhs
    for r in range(t.nrc):
        nf, nb = int(t.nf[r]), int(t.nb[r])
        typ = int(t.rate_type[r])
        ords = [t.ford[r, k] for k in range(nf)] + [t.bord[r, k] for k in range(nb)]
        npow = sum(1 for o in ords if o not in (1.0, 2.0))
        base = tr + 4                            # kf
        base += 2 * (nf + nb) + tr + 4          # Kc
        base += npow * tr + (nf + nb) + 2       # concentration products, q
        base += 2 * (nf + nb)                   # scatter into f
        jac = base
        jac += (nf * nf + nb * nb) + 2 * (nf + nb) * (nf + nb)
        jac += 12 + 2 * (nf + nb)
        if typ != 0:
            base += 2 * nsp
            jac += 2 * nsp + 3 * nsp * (nf + nb)
        if typ >= 2:
            base += 6 * tr + 20
            jac += 12 * tr + 60
        f_rhs += base
        f_jac += jac
    f_jac += 2.0 * nsp * nsp + 10.0 * nsp
    f_lu = 2.0 * (n ** 3 / 3.0 - n ** 2 / 2.0 + n / 6.0)
    f_solve = 2.0 * n * n
    return {"rhs": f_rhs, "jac": f_jac, "lu": f_lu, "solve": f_solve, "n": n,
            "transcendental": tr}


def work_flops(counters: Dict[str, int], fm: Dict[str, float]) -> float:
    """W = n_rhs F_rhs + n_jac F_jac + n_lu F_lu + n_newton F_solve."""
    return (counters["n_rhs"] * fm["rhs"] + counters["n_jac"] * fm["jac"] +
            counters["n_lu"] * fm["lu"] + counters["n_newton"] * fm["solve"])
