"""Seeded synthetic Chemkin mechanisms and cell states.

The reference solver reads a mechanism as three text files: a Chemkin
reaction file, an 80-column NASA-7 ("JANAF") thermo file and a free-format
transport file (chemistryRead/src/chemkinFileRead.cpp, JANAFThermoParsing.cpp,
JANAFTransportParsing.cpp). This module generates such mechanisms from a seed,
with the parameter distributions of the chemistry-source workloads:

* pre-exponential factor log-uniform in [1e8, 1e16] (cm, mol, s units as
  written to the file), temperature exponent uniform in [-1, 2], activation
  energy uniform in [0, 60] kcal/mol;
* element-balanced reactions (species are C/H/O/N formulas), a given number of
  third-body reactions and Troe fall-off reactions;
* NASA-7 two-range polynomials least-squares fitted to smooth seeded cp(T)
  curves, continuous in cp, h and s at the common temperature.

It also draws the seeded cell states (T, p, Y) of each workload. Everything
here is plain numpy; nothing depends on the reference at run time.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# Standard atomic weights used by the reference's element table
# (species/include/atomicWeights.hpp) for the elements the generator uses.
ATOMIC_WEIGHTS = {"H": 1.00797, "C": 12.01115, "N": 14.00670, "O": 15.99940}
ELEMENT_ORDER = ("C", "H", "O", "N")

PATM = 1.01325e5
RU_J_MOL_K = 1.380649e-23 * 6.02214076e23  # Boltzmann x Avogadro, J/(mol K)


@dataclasses.dataclass
class Species:
    name: str
    elements: Dict[str, int]
    t_low: float
    t_common: float
    t_high: float
    high: List[float]          # a1..a7 above t_common (cp/R basis)
    low: List[float]           # a1..a7 below t_common
    geometry: int              # 0 atom, 1 linear, 2 nonlinear
    eps_k: float               # Lennard-Jones well depth / kB [K]
    sigma: float               # collision diameter [Angstrom]
    dipole: float = 0.0
    polar: float = 0.0
    zrot: float = 1.0


@dataclasses.dataclass
class Reaction:
    reactants: List[Tuple[str, int]]
    products: List[Tuple[str, int]]
    A: float                    # cm-mol-s units, as written
    b: float
    Ea: float                   # cal/mol
    kind: str = "plain"         # plain | third_body | troe
    eff: Dict[str, float] = dataclasses.field(default_factory=dict)
    low: Optional[Tuple[float, float, float]] = None
    troe: Optional[Tuple[float, ...]] = None
    sri: Optional[Tuple[float, ...]] = None            # SRI a, b, c[, d, e] (replaces TROE)
    rev: Optional[Tuple[float, float, float]] = None   # REV A, b, Ea (cm-mol-s, cal/mol)
    ford: Dict[str, float] = dataclasses.field(default_factory=dict)
    rord: Dict[str, float] = dataclasses.field(default_factory=dict)
    units: Optional[str] = None                        # UNITS /.../ of this reaction
    plog: List[Tuple[float, float, float, float]] = dataclasses.field(default_factory=list)
    #                                                  # PLOG p [atm], A, b, Ea (cal/mol)
    activated: bool = False     # chemically activated: main line = low, HIGH = (A, b, Ea)
    lt: Optional[Tuple[float, float]] = None           # Landau-Teller B, C
    rlt: Optional[Tuple[float, float]] = None          # reverse Landau-Teller B, C (with rev)
    collision: bool = False                            # COLLEFF: A, b, Ea are the efficiency
    janev: Optional[Tuple[float, ...]] = None          # JAN b_0..b_8
    fit1: Optional[Tuple[float, ...]] = None           # FIT1 b_0..b_3


@dataclasses.dataclass
class Mechanism:
    species: List[Species]
    reactions: List[Reaction]
    seed: int
    units: Tuple[str, ...] = ()    # unit words on the REACTIONS line

    @property
    def names(self) -> List[str]:
        return [s.name for s in self.species]

    def weights(self) -> np.ndarray:
        return np.array([molecular_weight(s.elements) for s in self.species])


def molecular_weight(elements: Dict[str, int]) -> float:
    """Sum of n_atoms x atomic weight in the order the elements are written
    (species.cpp:92 accumulates the element list in file order)."""
    w = 0.0
    for el in ELEMENT_ORDER:
        n = elements.get(el, 0)
        if n:
            w += n * ATOMIC_WEIGHTS[el]
    return w


def formula_name(elements: Dict[str, int]) -> str:
    out = ""
    for el in ELEMENT_ORDER:
        n = elements.get(el, 0)
        if n == 1:
            out += el
        elif n > 1:
            out += f"{el}{n}"
    return out


# --------------------------------------------------------------------------
# thermo: smooth cp(T) curves fitted by two NASA-7 polynomials
# --------------------------------------------------------------------------

def _fit_nasa7(rng: np.random.Generator, natoms: int, linear: bool,
               h298_over_r: float, s298_over_r: float,
               t_low=300.0, t_common=1000.0, t_high=5000.0):
    """Fit both NASA-7 ranges to one smooth cp/R curve.

    cp/R(T) = c0 + (cinf - c0) * x^2/(1+x^2) with x = T/theta (a seeded,
    monotone saturating curve), sampled densely on each range. The high
    range is fitted with an equality constraint that makes cp continuous at
    t_common; h and s continuity then fix a6/a7 of both ranges."""
    if natoms == 1:
        c0, cinf = 2.5, 2.5 + rng.uniform(0.0, 0.3)
    else:
        c0 = 3.5 if (natoms == 2 or linear) else 4.0
        dof = 3 * natoms - (5 if (linear or natoms == 2) else 6)
        cinf = c0 + dof * rng.uniform(0.75, 1.0)
    theta = rng.uniform(600.0, 2500.0)

    def cp(T):
        x = T / theta
        return c0 + (cinf - c0) * x * x / (1.0 + x * x)

    def design(T):
        return np.stack([np.ones_like(T), T, T ** 2, T ** 3, T ** 4], axis=1)

    Tl = np.linspace(t_low, t_common, 200)
    Th = np.linspace(t_common, t_high, 400)
    lo = np.linalg.lstsq(design(Tl), cp(Tl), rcond=None)[0]
    # constrained LS for the high range: cp_high(t_common) == cp_low(t_common)
    Dh = design(Th)
    c = design(np.array([t_common]))[0]
    target = float(c @ lo)
    kkt = np.zeros((6, 6))
    kkt[:5, :5] = 2.0 * Dh.T @ Dh
    kkt[:5, 5] = c
    kkt[5, :5] = c
    rhs = np.concatenate([2.0 * Dh.T @ cp(Th), [target]])
    hi = np.linalg.solve(kkt, rhs)[:5]

    def h_poly(a, T):  # h/R without a6
        return a[0] * T + a[1] / 2 * T ** 2 + a[2] / 3 * T ** 3 + a[3] / 4 * T ** 4 + a[4] / 5 * T ** 5

    def s_poly(a, T):  # s/R without a7
        return a[0] * math.log(T) + a[1] * T + a[2] / 2 * T ** 2 + a[3] / 3 * T ** 3 + a[4] / 4 * T ** 4

    a6_lo = h298_over_r - h_poly(lo, 298.15)
    a7_lo = s298_over_r - s_poly(lo, 298.15)
    a6_hi = h_poly(lo, t_common) + a6_lo - h_poly(hi, t_common)
    a7_hi = s_poly(lo, t_common) + a7_lo - s_poly(hi, t_common)
    low = [float(x) for x in lo] + [float(a6_lo), float(a7_lo)]
    high = [float(x) for x in hi] + [float(a6_hi), float(a7_hi)]
    return low, high


def _species_pool(nsp: int, rng: np.random.Generator) -> List[Dict[str, int]]:
    base = [{"H": 2}, {"O": 2}, {"H": 1}, {"O": 1}, {"H": 1, "O": 1},
            {"H": 2, "O": 1}, {"H": 1, "O": 2}, {"H": 2, "O": 2}, {"N": 2}]
    if nsp <= len(base):
        return base[:nsp]
    pool = []
    for c in range(0, 3):
        for h in range(0, 7):
            for o in range(0, 4):
                for n in range(0, 3):
                    tot = c + h + o + n
                    if tot == 0 or tot > 8:
                        continue
                    el = {k: v for k, v in (("C", c), ("H", h), ("O", o), ("N", n)) if v}
                    if el in base:
                        continue
                    pool.append(el)
    extra = [pool[i] for i in rng.permutation(len(pool))]
    # make sure the carbon / nitrogen atoms and their diatomics exist
    must = [{"C": 1}, {"N": 1}, {"C": 1, "O": 1}, {"C": 1, "O": 2}, {"N": 1, "O": 1},
            {"C": 1, "H": 4}, {"C": 1, "H": 3}, {"C": 1, "H": 2, "O": 1}]
    rest = [e for e in extra if e not in must]
    out = base + must + rest
    return out[:nsp]


def _element_vec(el: Dict[str, int]) -> Tuple[int, ...]:
    return tuple(el.get(e, 0) for e in ELEMENT_ORDER)


def make_mechanism(nsp: int, nrc: int, n_third_body: int, n_troe: int,
                   seed: int) -> Mechanism:
    """Seeded synthetic mechanism with nsp species and nrc reversible
    Arrhenius reactions, n_third_body of them '+M' and n_troe of them Troe
    fall-off '(+M)'. The last species is an inert diluent (N2 for the small
    mechanism) unless it takes part in a drawn reaction."""
    rng = np.random.default_rng(seed)
    els = _species_pool(nsp, rng)
    species: List[Species] = []
    for el in els:
        natoms = sum(el.values())
        linear = natoms <= 2
        name = formula_name(el)
        elemental = (len(el) == 1 and natoms == 2)
        if elemental:
            h298 = 0.0
        elif natoms == 1:
            h298 = rng.uniform(12000.0, 25000.0)      # atoms: h/R in K (100-210 kJ/mol)
        else:
            h298 = rng.uniform(-8000.0, 4000.0)       # h/R in K (-67..+33 kJ/mol)
        s298 = rng.uniform(13.0, 18.0) + 2.5 * natoms
        low, high = _fit_nasa7(rng, natoms, linear, h298, s298)
        geom = 0 if natoms == 1 else (1 if linear else 2)
        eps = rng.uniform(30.0, 500.0)
        sigma = rng.uniform(2.0, 4.5) + 0.15 * natoms
        dip = 0.0 if rng.uniform() < 0.7 else rng.uniform(0.5, 2.0)
        pol = rng.uniform(0.5, 3.0) if natoms > 1 else 0.0
        zr = rng.uniform(0.0, 4.0) if natoms > 1 else 0.0
        species.append(Species(name, el, 300.0, 1000.0, 5000.0, high, low,
                               geom, float(eps), float(sigma), float(dip),
                               float(pol), float(zr)))

    vec = [np.array(_element_vec(s.elements)) for s in species]
    idx_of = {_element_vec(s.elements): i for i, s in enumerate(species)}
    # candidates: A+B=C+D (exchange) and A+B=C (recombination)
    pair_sum: Dict[Tuple[int, ...], List[Tuple[int, int]]] = {}
    for i in range(nsp):
        for j in range(i, nsp):
            key = tuple(vec[i] + vec[j])
            pair_sum.setdefault(key, []).append((i, j))
    exchange = []
    for key, pairs in pair_sum.items():
        for a in range(len(pairs)):
            for b in range(a + 1, len(pairs)):
                (i, j), (k, m) = pairs[a], pairs[b]
                if not ({i, j} & {k, m}):
                    exchange.append(((i, j), (k, m)))
    recomb = []
    for key, pairs in pair_sum.items():
        if key in idx_of:
            c = idx_of[key]
            for (i, j) in pairs:
                if c not in (i, j):
                    recomb.append(((i, j), (c,)))
    rng.shuffle(exchange)
    rng.shuffle(recomb)
    n_recomb = n_third_body + n_troe
    if len(recomb) < n_recomb or len(exchange) < nrc - n_recomb:
        raise ValueError("species pool too small for the requested reactions")

    def draw_arrhenius():
        return (10.0 ** rng.uniform(8.0, 16.0), rng.uniform(-1.0, 2.0),
                rng.uniform(0.0, 60.0) * 1000.0)

    def pick(cands, n, used):
        # cover species that no reaction touches yet first
        out = []
        touched = set(s for r in used for s in r[0] + r[1])
        for cand in cands:
            if len(out) == n:
                break
            sp = set(cand[0] + cand[1])
            if cand in used or cand in out:
                continue
            if sp - touched or len(touched) >= nsp - 1:
                out.append(cand)
                touched |= sp
        for cand in cands:
            if len(out) == n:
                break
            if cand not in out and cand not in used:
                out.append(cand)
        return out

    rec_sel = pick(recomb, n_recomb, [])
    exc_sel = pick(exchange, nrc - n_recomb, rec_sel)
    names = [s.name for s in species]

    def side(ids):
        out: Dict[str, int] = {}
        for i in ids:
            out[names[i]] = out.get(names[i], 0) + 1
        return list(out.items())

    reactions: List[Reaction] = []
    for (lhs, rhs) in exc_sel:
        A, b, Ea = draw_arrhenius()
        reactions.append(Reaction(side(lhs), side(rhs), A, b, Ea, "plain"))
    for n, (lhs, rhs) in enumerate(rec_sel):
        A, b, Ea = draw_arrhenius()
        # third-body efficiencies on up to 3 species
        ne = int(rng.integers(1, 4))
        eff_idx = rng.choice(nsp, size=min(ne, nsp), replace=False)
        eff = {names[i]: float(np.round(rng.uniform(0.3, 6.0), 2)) for i in eff_idx}
        if n < n_third_body:
            reactions.append(Reaction(side(lhs), side(rhs), A, b, Ea, "third_body", eff))
        else:
            A0, b0, E0 = draw_arrhenius()
            troe = (float(np.round(rng.uniform(0.1, 0.9), 4)),
                    float(np.round(rng.uniform(30.0, 500.0), 1)),
                    float(np.round(rng.uniform(500.0, 3000.0), 1)),
                    float(np.round(rng.uniform(2000.0, 8000.0), 1)))
            reactions.append(Reaction(side(lhs), side(rhs), A, b, Ea, "troe", eff,
                                      (A0, b0, E0), troe))
    order = rng.permutation(len(reactions))
    reactions = [reactions[i] for i in order]
    return Mechanism(species, reactions, seed)


def extended_mechanism(seed: int = 20241117) -> Mechanism:
    """9 species / 21 reactions using every rate form the reader takes beyond
    the small mechanism's: two SRI fall-off reactions (3 and 5 parameters) and
    one Troe, explicit reverse parameters (REV) on two Arrhenius and one
    third-body reaction, a forward and a reverse order override (FORD 1.5,
    RORD 1.5), energies written in kJ/mol on the REACTIONS line, and
    per-reaction UNITS (molecules for one reaction, kcal/mol for another),
    three PLOG pressure tables, a chemically activated (HIGH) reaction and a
    Landau-Teller (LT) one.
    The rate parameters stay those of the drawn mechanism; the file carries
    them in the declared units. (Orders below one give rates that are not
    Lipschitz at zero concentration; with such an order this mechanism's
    cells answer one-ulp input changes with 1e-6 changes of T, which no
    parity tolerance between two libms survives, so both overrides are 1.5.)"""
    m = make_mechanism(9, 21, 3, 3, seed)
    rng = np.random.default_rng(seed + 1)
    m.units = ("KJOU", "MOLES")
    fall = [r for r in m.reactions if r.kind == "troe"]
    fall[0].sri = (float(np.round(rng.uniform(0.5, 2.0), 4)),
                   float(np.round(rng.uniform(100.0, 800.0), 1)),
                   float(np.round(rng.uniform(500.0, 2000.0), 1)))
    fall[0].troe = None
    fall[1].sri = (float(np.round(rng.uniform(0.5, 2.0), 4)),
                   float(np.round(rng.uniform(100.0, 800.0), 1)),
                   float(np.round(rng.uniform(500.0, 2000.0), 1)),
                   float(np.round(rng.uniform(0.8, 1.2), 4)),
                   float(np.round(rng.uniform(-0.3, 0.3), 4)))
    fall[1].troe = None
    fall[1].activated = True     # chemically activated bimolecular (HIGH) with the SRI form
    plain = [r for r in m.reactions if r.kind == "plain"]
    tb = [r for r in m.reactions if r.kind == "third_body"]

    def draw_rev():
        return (10.0 ** rng.uniform(9.0, 13.0), float(np.round(rng.uniform(-0.8, 0.8), 4)),
                float(np.round(rng.uniform(0.0, 40.0), 3)) * 1000.0)

    plain[0].rev = draw_rev()
    plain[1].rev = draw_rev()
    tb[0].rev = draw_rev()
    plain[2].ford = {plain[2].reactants[0][0]: 1.5}
    plain[3].rord = {plain[3].products[0][0]: 1.5}
    plain[4].units = "MOLEC"
    plain[5].units = "KCAL"
    # pressure tables: cells at 1-5 atm fall inside the first (interpolated),
    # above the second and below the third (whose lowest pressure is listed
    # twice, the two rates adding up)
    for r, ps in ((plain[6], (0.1, 1.0, 10.0)), (plain[7], (0.01, 0.1, 0.5)),
                  (plain[8], (10.0, 10.0, 100.0))):
        r.plog = [(pa, float(r.A * 10.0 ** rng.uniform(-1.0, 1.0)),
                   float(np.round(r.b + rng.uniform(-0.2, 0.2), 6)),
                   float(np.round(r.Ea + rng.uniform(-2000.0, 2000.0), 4))) for pa in ps]
    plain[9].lt = (float(np.round(rng.uniform(-20.0, 20.0), 4)),
                   float(np.round(rng.uniform(-50.0, 50.0), 4)))
    return m


def fitted_rates_mechanism(seed: int = 20240901,
                           collision: Tuple[float, float, float] = (2e-21, 0.0, 0.0)) -> Mechanism:
    """The small mechanism with one reaction on a Janev rate (JAN, nine
    coefficients of powers of ln T) and one on a power-series rate (FIT1,
    four coefficients of powers of 1/T), small enough to keep the rates within
    a decade or so of the drawn Arrhenius ones, one Landau-Teller reaction
    with explicit reverse parameters in the Landau-Teller form (LT, REV, RLT),
    and one collision-efficiency reaction (COLLEFF) with efficiency A, b, Ea
    `collision`. With b = Ea = 0 the reference's dk/dT of that reaction is zero;
    otherwise it is the Arrhenius derivative times dZ/dT, about 1e25 times the
    rate's own derivative, which stalls the Newton iterations, so integrations
    use the default and only rate and Jacobian checks use other values."""
    m = small_mechanism(seed)
    rng = np.random.default_rng(seed + 7)
    plain = [r for r in m.reactions if r.kind == "plain"]
    plain[0].janev = tuple(float(np.round(rng.uniform(-1.0, 1.0) * 0.3 / 8.0 ** n, 10))
                           for n in range(9))
    plain[1].fit1 = (float(np.round(rng.uniform(-300.0, 300.0), 4)),
                     float(np.round(rng.uniform(-1e5, 1e5), 2)),
                     float(np.round(rng.uniform(-1e7, 1e7), 1)),
                     float(np.round(rng.uniform(-1e9, 1e9), 1)))
    plain[2].lt = (float(np.round(rng.uniform(-20.0, 20.0), 4)),
                   float(np.round(rng.uniform(-50.0, 50.0), 4)))
    plain[2].rev = (float(10.0 ** np.round(rng.uniform(9.0, 13.0), 3)),
                    float(np.round(rng.uniform(-0.8, 0.8), 4)),
                    float(np.round(rng.uniform(0.0, 40.0), 3)) * 1000.0)
    plain[2].rlt = (float(np.round(rng.uniform(-20.0, 20.0), 4)),
                    float(np.round(rng.uniform(-50.0, 50.0), 4)))
    plain[3].collision = True
    plain[3].A, plain[3].b, plain[3].Ea = collision
    return m


def small_mechanism(seed: int = 20240901) -> Mechanism:
    """9 species / 21 reversible Arrhenius reactions, 3 third-body, 1 Troe."""
    return make_mechanism(9, 21, 3, 1, seed)


def large_mechanism(seed: int = 20240953) -> Mechanism:
    """53 species / 325 reactions, 15% third-body (49), 5% Troe (16)."""
    return make_mechanism(53, 325, 49, 16, seed)


# --------------------------------------------------------------------------
# file writers (Chemkin / NASA-7 80 column / transport)
# --------------------------------------------------------------------------

def _fmt_e(x: float) -> str:
    # E15.8 field, as in the NASA-7 format
    return f"{x:15.8E}"


def _reaction_side(side: Sequence[Tuple[str, int]], kind: str) -> str:
    terms = [(f"{n}{s}" if n > 1 else s) for s, n in side]
    txt = "+".join(terms)
    if kind == "third_body":
        txt += "+M"
    elif kind == "troe":
        txt += "(+M)"
    return txt


def _energy_in(ea_cal: float, unit: str) -> float:
    """An activation energy given in cal/mol, expressed in `unit`."""
    if unit in ("CAL", "CAL/MOLE"):
        return ea_cal
    if unit in ("KCAL", "KCAL/MOLE"):
        return ea_cal / 1000.0
    if unit in ("JOUL", "JOULES/MOLE"):
        return ea_cal * 4.184
    if unit in ("KJOU", "KJOULES/MOLE"):
        return ea_cal * 4.184 / 1000.0
    if unit in ("KELV", "KELVINS"):
        return ea_cal / (1.380649e-23 * 6.02214076e23 / 4.184)
    raise ValueError(unit)


def _pre_exp_in(a_mol: float, order: float, third: bool, unit: str) -> float:
    """A pre-exponential factor in mol-cm-s units, expressed per molecule when
    `unit` says MOLEC (the reader multiplies by NA^(order - 1), or NA^order
    for a reaction with a third body)."""
    if not unit.startswith("MOLEC"):
        return a_mol
    return a_mol / 6.02214076e23 ** (order if third else order - 1.0)


def write_chemkin(mech: Mechanism, out_dir: str, stem: str = "mech") -> Tuple[str, str, str]:
    os.makedirs(out_dir, exist_ok=True)
    che = os.path.join(out_dir, f"{stem}.che")
    thermo = os.path.join(out_dir, f"{stem}_thermo.dat")
    tran = os.path.join(out_dir, f"{stem}_transport.dat")
    used_el = [e for e in ELEMENT_ORDER if any(e in s.elements for s in mech.species)]
    lines = ["! seeded synthetic mechanism, seed %d" % mech.seed, "ELEMENTS",
             " ".join(used_el), "END", "SPECIES"]
    names = mech.names
    for i in range(0, len(names), 8):
        lines.append(" ".join(names[i:i + 8]))
    lines += ["END", "REACTIONS" + "".join(" " + u for u in mech.units)]
    g_A = next((u for u in mech.units if u.startswith("MOLEC")), "MOLES")
    g_E = next((u for u in mech.units if not u.startswith("MOLE")), "CAL")
    for r in mech.reactions:
        u_A = r.units if (r.units or "").startswith("MOLEC") else g_A
        u_E = r.units if (r.units and not r.units.startswith("MOLE")) else g_E
        E = lambda ea: _energy_in(ea, u_E)
        fo = sum(r.ford.get(s_, n) for s_, n in r.reactants)
        bo = sum(r.rord.get(s_, n) for s_, n in r.products)
        third = r.kind != "plain"
        A = lambda a, o: _pre_exp_in(a, o, third, u_A)
        eq = _reaction_side(r.reactants, r.kind) + "=" + _reaction_side(r.products, r.kind)
        if r.activated:
            A0, b0, E0 = r.low
            lines.append(f"{eq}   {A(A0, fo):.6E}  {b0:.6f}  {E(E0):.4f}")
            lines.append(f"   HIGH / {A(r.A, fo):.6E}  {r.b:.6f}  {E(r.Ea):.4f} /")
        else:
            lines.append(f"{eq}   {A(r.A, fo):.6E}  {r.b:.6f}  {E(r.Ea):.4f}")
        if r.kind == "troe" and not r.activated:
            A0, b0, E0 = r.low
            lines.append(f"   LOW / {A(A0, fo):.6E}  {b0:.6f}  {E(E0):.4f} /")
        if r.kind == "troe":
            if r.sri is not None:
                lines.append("   SRI / " + "  ".join(f"{x:.6g}" for x in r.sri) + " /")
            else:
                lines.append("   TROE / " + "  ".join(f"{x:.6g}" for x in r.troe) + " /")
        if r.kind in ("third_body", "troe") and r.eff:
            lines.append("   " + " ".join(f"{k}/{v:.2f}/" for k, v in r.eff.items()))
        if r.rev is not None:
            Ar, br, Er = r.rev
            lines.append(f"   REV / {A(Ar, bo):.6E}  {br:.6f}  {E(Er):.4f} /")
        for k, v in r.ford.items():
            lines.append(f"   FORD / {k} {v:g} /")
        for k, v in r.rord.items():
            lines.append(f"   RORD / {k} {v:g} /")
        if r.units:
            lines.append(f"   UNITS / {r.units} /")
        for pa, Ap, bp, Ep in r.plog:
            lines.append(f"   PLOG / {pa:g}  {A(Ap, fo):.6E}  {bp:.6f}  {E(Ep):.4f} /")
        if r.lt is not None:
            lines.append(f"   LT / {r.lt[0]:g}  {r.lt[1]:g} /")
        if r.rlt is not None:
            lines.append(f"   RLT / {r.rlt[0]:g}  {r.rlt[1]:g} /")
        if r.collision:
            lines.append("   COLLEFF")
        if r.janev is not None:
            lines.append("   JAN / " + "  ".join(f"{x:.10g}" for x in r.janev) + " /")
        if r.fit1 is not None:
            lines.append("   FIT1 / " + "  ".join(f"{x:.10g}" for x in r.fit1) + " /")
    lines += ["END", ""]
    with open(che, "w") as f:
        f.write("\n".join(lines))

    tl = ["THERMO", "   300.000  1000.000  5000.000"]
    for s in mech.species:
        elfield = ""
        for e in ELEMENT_ORDER:
            if e in s.elements:
                elfield += f"{e:<2}{s.elements[e]:>3}"
        elfield = f"{elfield:<20}"[:20]
        l1 = f"{s.name:<18}{'SYNTH':<6}{elfield}G{s.t_low:10.3f}{s.t_high:10.3f}{s.t_common:8.2f}"
        l1 = f"{l1:<79}1"
        h, lo = s.high, s.low
        l2 = "".join(_fmt_e(x) for x in h[0:5]) + "    2"
        l3 = "".join(_fmt_e(x) for x in (h[5], h[6], lo[0], lo[1], lo[2])) + "    3"
        l4 = "".join(_fmt_e(x) for x in (lo[3], lo[4], lo[5], lo[6])) + "                   4"
        tl += [l1, l2, l3, l4]
    tl += ["END", ""]
    with open(thermo, "w") as f:
        f.write("\n".join(tl))

    trl = []
    for s in mech.species:
        trl.append(f"{s.name:<18}{s.geometry:>2}{s.eps_k:10.3f}{s.sigma:10.3f}"
                   f"{s.dipole:10.3f}{s.polar:10.3f}{s.zrot:10.3f}")
    trl.append("")
    with open(tran, "w") as f:
        f.write("\n".join(trl))
    return che, thermo, tran


# --------------------------------------------------------------------------
# cell states
# --------------------------------------------------------------------------

@dataclasses.dataclass
class Cells:
    T: np.ndarray      # [n]
    p: np.ndarray      # [n] Pa
    Y: np.ndarray      # [nsp, n] structure of arrays

    @property
    def n(self) -> int:
        return int(self.T.shape[0])


def dirichlet_cells(nsp: int, n: int, seed: int, T_range=(1000.0, 2500.0),
                    p_atm_range=(1.0, 5.0), alpha=0.5) -> Cells:
    """T uniform, p uniform in atm, Y ~ Dirichlet(alpha) over all species."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(T_range[0], T_range[1], n)
    p = rng.uniform(p_atm_range[0], p_atm_range[1], n) * PATM
    Y = rng.dirichlet(np.full(nsp, alpha), n).T.copy()
    return Cells(T, p, np.ascontiguousarray(Y))


def ignition_cells(nsp: int, n: int, seed: int, reactant_idx: Sequence[int],
                   T_range=(1100.0, 1300.0), p_atm_range=(1.0, 5.0), alpha=2.0) -> Cells:
    """Near-ignition cells: T in T_range, Y ~ Dirichlet(alpha) over the
    reactant species only (all other species zero)."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(T_range[0], T_range[1], n)
    p = rng.uniform(p_atm_range[0], p_atm_range[1], n) * PATM
    Y = np.zeros((nsp, n))
    Y[list(reactant_idx), :] = rng.dirichlet(np.full(len(reactant_idx), alpha), n).T
    return Cells(T, p, Y)


def mixture_density(mech_W: np.ndarray, cells: Cells) -> np.ndarray:
    """Perfect-gas density rho = p / (Rm T), Rm = Ru / Wmean,
    Wmean = 1 / sum_i(Y_i / W_i)."""
    ru = RU_J_MOL_K * 1e3
    s = np.zeros(cells.n)
    for i in range(cells.Y.shape[0]):
        s += cells.Y[i] / mech_W[i]
    Rm = ru / (1.0 / np.maximum(s, 1e-300))
    return cells.p / (Rm * cells.T)
