"""Mechanism reader and compiler: Chemkin + NASA-7 + transport -> flat tables.

This is the host-side half of the drop-in boundary. It reads the three text
files the reference reads (chemistryRead/src/chemkinFileRead.cpp,
JANAFThermoParsing.cpp, JANAFTransportParsing.cpp) and produces the flat,
structure-of-arrays tables that the C ABI (`hc_mech_create`, declared in
include/hurchem_b200.h) uploads to the GPU. Unit conversions and derived
constants are computed with the same floating-point operations, in the same
order, as the reference so that the tables hold identical bits:

* R = kB * NA [J/mol/K], Ru = R * 1e3 [J/kmol/K]
  (Hurricane/common/constants/physicalConstant.hpp:158,183);
* W_i = sum of n_atoms * atomic weight in file order (species.cpp:92);
  R_i = Ru / W_i;
* NASA-7 coefficients are converted to the mass basis, a_k * R_i
  (thermo/src/JANAF.cpp:44-58);
* A is scaled by pow(1e-3, order - 1) with order = sum of forward orders, an
  extra 1e-3 for '+M' third-body reactions and for the low-pressure limit of
  fall-off reactions; E [cal/mol] becomes Ta = E / (R / 4.184)
  (chemkinFileRead.cpp:1374-1455, :1654-1696);
* the species of each side are held in a name-sorted map, repeated species
  merged (chemkinFileRead.cpp:902-925), so the forward/backward coefficient
  lists are in lexicographic name order;
* third-body efficiencies default to 1.0 for every species
  (chemkinFileRead.cpp:1050-1061, :1063-1085).

* units: the REACTIONS line may name the units of A (MOLES, MOLECULES) and
  of E (CAL/MOLE, KCAL/MOLE, JOULES/MOLE, KJOULES/MOLE, KELVINS, EVOLTS),
  and a reaction may override them with UNITS /.../; the factors are those
  of chemkinFileRead::changeUnit (chemkinFileRead.cpp:1654-1696), with the
  order of a side taken from its reaction orders (after FORD / RORD).

Supported rate forms: Arrhenius, Arrhenius third-body (+M), unimolecular
fall-off (+M, or a named third body +X) with Lindemann, Troe (3 or 4
parameters) or SRI (3 or 5 parameters); reversible (=, <=>) and irreversible (=>) reactions; explicit
reverse Arrhenius parameters (REV, reversibleReactionWithRevPars) on
Arrhenius and third-body reactions; non-stoichiometric orders (FORD, RORD).
pressure-dependent Arrhenius tables (PLOG, logInterpolationRR) on reactions
without a third body; chemically activated bimolecular reactions (HIGH,
chemicallyActicatedBimolecularRR) with any fall-off function; Landau-Teller
rates (LT, LandauTellerRR), with REV also in the reverse direction (RLT);
Janev (JAN, JanevRR), power-series (FIT1, powerSeriesRR) and collision-
efficiency (COLLEFF, collisionRR) rates. TDEP, XSMI, MOME and EXCI, which the
reference's reader refuses too, are rejected with NotImplementedError, and
so is CHEB, whose reference implementation does not evaluate the Chebyshev
fit (see parse_chemkin).
"""
from __future__ import annotations

import dataclasses
import math
import re
from typing import Dict, List, Optional, Tuple

import numpy as np

# physical constants, evaluated exactly as the reference's constexprs
KB = 1.380649e-23
NA = 6.02214076e23
R_J_MOL_K = KB * NA
RU = R_J_MOL_K * 1e3
PATM = 1.01325e5
CAL_TH = 4.184

# element table entries for the elements that may appear (standard atomic
# weights; species/include/atomicWeights.hpp holds the same numbers)
ATOMIC_WEIGHTS = {
    "H": 1.00797, "D": 2.01410, "HE": 4.00260, "C": 12.01115, "N": 14.00670,
    "O": 15.99940, "F": 18.99840, "NE": 20.18300, "S": 32.06400, "CL": 35.45300,
    "AR": 39.94800,
}

MAX_SIDE = 4          # species per reaction side held in the flat tables

# rate-law codes of the flat tables
RATE_ARRHENIUS = 0
RATE_THIRD_BODY = 1
RATE_LINDEMANN = 2
RATE_TROE3 = 3
RATE_TROE4 = 4
RATE_SRI = 5
RATE_PLOG = 6
RATE_LANDAU_TELLER = 7
RATE_JANEV = 8
RATE_POWER_SERIES = 9
RATE_COLLISION = 10

# reversibility codes
IRREVERSIBLE = 0
REVERSIBLE = 1
REVERSIBLE_REV = 2     # explicit reverse Arrhenius parameters

# Chemkin unit keywords (chemkinFileRead.cpp:45-73)
UNITS_A = {"MOLE": "MOLES", "MOLES": "MOLES", "MOLEC": "MOLECULES", "MOLECULE": "MOLECULES",
           "MOLECULES": "MOLECULES"}
UNITS_E = {"CAL": "CAL", "CAL/MOLE": "CAL", "EVOL": "EVOL", "EVOLTS": "EVOL", "JOUL": "JOUL",
           "JOULES/MOLE": "JOUL", "KCAL": "KCAL", "KCAL/MOLE": "KCAL", "KELV": "KELV",
           "KELVINS": "KELV", "KJOU": "KJOU", "KJOULES/MOLE": "KJOU"}
ELECTRON_VOLT = 1.6021766208e-19    # J (physicalConstant.hpp:59,114)
# auxiliary keywords that the reference's own reader refuses as not yet supported
# (chemkinFileRead.cpp:530-558)
_UNSUPPORTED_AUX = {"TDEP", "XSMI", "MOME", "EXCI"}


@dataclasses.dataclass
class ParsedReaction:
    fwd: List[Tuple[int, float]]      # (species index, stoich) name-sorted
    bwd: List[Tuple[int, float]]
    reversible: bool
    A: float
    b: float
    E: float
    kind: str                         # arrhenius | third_body | falloff
    eff: Optional[np.ndarray] = None
    low: Optional[Tuple[float, float, float]] = None
    troe: Optional[List[float]] = None
    sri: Optional[List[float]] = None
    rev: Optional[Tuple[float, float, float]] = None
    ford: Optional[Dict[int, float]] = None     # species -> forward order (FORD)
    rord: Optional[Dict[int, float]] = None     # species -> reverse order (RORD)
    units_A: str = "MOLES"
    units_E: str = "CAL"
    plog: Optional[List[Tuple[float, float, float, float]]] = None   # (p atm, A, b, E) as read
    high: Optional[Tuple[float, float, float]] = None   # HIGH A, b, E (chemically activated)
    lt: Optional[Tuple[float, float]] = None             # Landau-Teller B, C
    rlt: Optional[Tuple[float, float]] = None            # reverse Landau-Teller B, C (RLT)
    collision: bool = False                              # COLLEFF: collision efficiency
    named_third: Optional[int] = None                    # species of a (+X) third body
    janev: Optional[List[float]] = None                  # JAN b_0..b_8
    fit1: Optional[List[float]] = None                   # FIT1 b_0..b_3


@dataclasses.dataclass
class MechTables:
    """Flat tables in SI units (kmol, m^3, s, K, J, kg)."""
    names: List[str]
    W: np.ndarray            # [nsp]
    Ri: np.ndarray           # [nsp]
    Trange: np.ndarray       # [nsp, 3] Tlow, Tcommon, Thigh
    nasa: np.ndarray         # [nsp, 2, 7] mass basis: [low, high]
    elem_names: List[str]
    elem_matrix: np.ndarray  # [nelem, nsp] atoms per species
    rate_type: np.ndarray    # [nrc] int32
    reversible: np.ndarray   # [nrc] int32
    arr: np.ndarray          # [nrc, 3] A, beta, Ta (high-pressure limit for fall-off)
    arr0: np.ndarray         # [nrc, 3] low-pressure limit (fall-off only)
    troe: np.ndarray         # [nrc, 4] alpha, T***, T*, T**
    eff: np.ndarray          # [nrc, nsp] third-body efficiencies (1.0 unused rows)
    nf: np.ndarray           # [nrc] int32
    nb: np.ndarray           # [nrc] int32
    fidx: np.ndarray         # [nrc, MAX_SIDE] int32
    bidx: np.ndarray
    fnu: np.ndarray          # [nrc, MAX_SIDE] stoichiometric coefficients
    bnu: np.ndarray
    ford: np.ndarray         # [nrc, MAX_SIDE] reaction orders
    bord: np.ndarray
    sum_stoi: np.ndarray     # [nrc] sum(bnu) - sum(fnu)
    # transport (kinetic theory)
    geom: np.ndarray         # [nsp] int32
    eps_k: np.ndarray        # [nsp]
    sigma: np.ndarray        # [nsp]
    dipole: np.ndarray
    polar: np.ndarray
    zrot: np.ndarray
    sri: Optional[np.ndarray] = None       # [nrc, 5] a, b, c, d, e (SRI fall-off)
    arr_rev: Optional[np.ndarray] = None   # [nrc, 3] explicit reverse A, beta, Ta (REV)
    plog_ptr: Optional[np.ndarray] = None  # [nrc + 1] int32 entries of each PLOG reaction
    plog_p: Optional[np.ndarray] = None    # [n] Pa, sorted per reaction
    plog_arr: Optional[np.ndarray] = None  # [n, 3] A, beta, Ta
    activated: Optional[np.ndarray] = None  # [nrc] int32 1: chemically activated (HIGH)
    lt: Optional[np.ndarray] = None        # [nrc, 2] Landau-Teller B, C
    xcoef: Optional[np.ndarray] = None     # [nrc, 9] Janev b_0..b_8 / power-series b_0..b_3

    @property
    def nsp(self) -> int:
        return len(self.names)

    @property
    def nrc(self) -> int:
        return int(self.rate_type.shape[0])


def _strip_comments(text: str) -> str:
    return "\n".join(line.split("!", 1)[0] for line in text.splitlines())


def _section(text: str, start_re: str) -> str:
    m = re.search(start_re + r"\s+([\s\S]*?)\s+END", text, re.IGNORECASE)
    return m.group(1) if m else ""


def _read_real(s: str) -> float:
    s = s.strip().replace("D", "E").replace("d", "e")
    return float(s)


def _parse_side(txt: str, index: Dict[str, int]) -> List[Tuple[int, float]]:
    counts: Dict[str, float] = {}
    for term in txt.split("+"):
        term = term.strip()
        if not term:
            continue
        m = re.match(r"^((?:[0-9]*)\.*[0-9]*)\s*(\S+)$", term)
        coef = float(m.group(1)) if m.group(1) else 1.0
        name = m.group(2)
        counts[name] = counts.get(name, 0.0) + coef
    out = []
    for name in sorted(counts):           # std::map order
        if name not in index:
            raise ValueError(f"unknown species {name!r}")
        out.append((index[name], counts[name]))
    return out


def _split_side_terms(side: str) -> str:
    # '+' signs that separate species (a leading '+' of a charge is not used here)
    return side


def _unit(word: str, where: str) -> Tuple[str, str]:
    w = word.strip().upper()
    if w in UNITS_A:
        return "A", UNITS_A[w]
    if w in UNITS_E:
        return "E", UNITS_E[w]
    raise ValueError(f"unknown unit {word!r} {where}")


def change_unit(order: float, units_A: str, units_E: str, third_body: bool) -> Tuple[float, float]:
    """(A factor, E factor) of chemkinFileRead::changeUnit (chemkinFileRead.cpp:1654-1696):
    A [units_A, cm, s] -> [kmol, m^3, s] for a side of total order `order`,
    and the divisor that turns E [units_E] into an activation temperature."""
    RRjoule = R_J_MOL_K
    RRcal = RRjoule / CAL_TH
    if units_A == "MOLECULES":
        Af = math.pow(NA, order) if third_body else math.pow(NA, order - 1.0)
        Af *= math.pow(0.001, order - 1.0)
    else:
        Af = math.pow(0.001, order - 1.0)
    Ef = {"CAL": RRcal, "KCAL": RRcal / 1000.0, "EVOL": RRjoule / ELECTRON_VOLT,
          "JOUL": RRjoule, "KJOU": RRjoule / 1000.0, "KELV": 1.0}[units_E]
    return Af, Ef


_AUX_RE = re.compile(r"(\S+?)\s*/\s*([^/]*?)\s*/|(\S+)")


def parse_chemkin(che_text: str, species_names: Optional[List[str]] = None):
    text = _strip_comments(che_text)
    sp_txt = _section(text, r"SPEC(?:|IE|IES)")
    names = species_names or sp_txt.split()
    index = {n: i for i, n in enumerate(names)}
    el_txt = _section(text, r"ELEM(?:|ENT|ENTS)")
    elements = [e.upper() for e in el_txt.split()]
    # REACTIONS [units of A] [units of E] on its own line, then the reactions
    # up to END (chemkinFileRead.cpp:1197-1284 for the units)
    m = re.search(r"\bREAC(?:TIONS|TION|)\b([^\n]*)\n([\s\S]*?)(?:^|\n)[ \t]*END\b", text,
                  re.IGNORECASE | re.MULTILINE)
    header, rx_txt = (m.group(1), m.group(2)) if m else ("", "")
    units = {"A": "MOLES", "E": "CAL"}
    for word in header.split():
        kind, u = _unit(word, "on the REACTIONS line")
        units[kind] = u
    lines = [l for l in rx_txt.splitlines() if l.strip()]
    line_re = re.compile(r"^(.*?)\s*(<=>|=>|=)\s*(.*?)\s+([-+]?[0-9.]+(?:[eEdD][-+]?[0-9]+)?)"
                         r"\s+(\S+)\s+(\S+)\s*$")
    reactions: List[ParsedReaction] = []
    cur: Optional[ParsedReaction] = None
    for line in lines:
        m = line_re.match(line.strip())
        if m and ("=" in m.group(2)) and "/" not in m.group(1):
            lhs, arrow, rhs = m.group(1), m.group(2), m.group(3)
            A, b, E = _read_real(m.group(4)), _read_real(m.group(5)), _read_real(m.group(6))
            kind = "arrhenius"
            pd = re.compile(r"\(\s*\+\s*(\S+?)\s*\)")
            third = None
            if pd.search(lhs) or pd.search(rhs):
                tl, tr = pd.search(lhs), pd.search(rhs)
                if not (tl and tr) or tl.group(1) != tr.group(1):
                    raise ValueError(f"pressure-dependent reaction with unmatched third bodies: "
                                     f"{line.strip()!r}")
                third = tl.group(1)
                if third.upper() != "M" and third not in index:
                    raise ValueError(f"third body {third!r} is not a species")
                lhs, rhs = pd.sub("", lhs), pd.sub("", rhs)
                kind = "falloff"
            tb = re.compile(r"\+\s*M(?![-a-zA-Z0-9])", re.IGNORECASE)
            if tb.search(lhs) or tb.search(rhs):
                lhs, rhs = tb.sub("", lhs), tb.sub("", rhs)
                kind = "third_body"
            cur = ParsedReaction(_parse_side(lhs, index), _parse_side(rhs, index),
                                 arrow != "=>", A, b, E, kind,
                                 units_A=units["A"], units_E=units["E"])
            if kind in ("third_body", "falloff"):
                cur.eff = np.ones(len(names))
            if third is not None and third.upper() != "M":
                # a named third body (+X): efficiency 1 for X, 0 for every other
                # species (chemkinFileRead.cpp:1002-1061); an efficiency line may
                # then name X only (chemkinFileRead.cpp:797-822)
                cur.eff = np.zeros(len(names))
                cur.eff[index[third]] = 1.0
                cur.named_third = index[third]
            reactions.append(cur)
            continue
        # auxiliary line: KEY / values / groups, bare words, species efficiencies
        if cur is None:
            raise ValueError(f"auxiliary data before the first reaction: {line.strip()!r}")
        for key, val, word in _AUX_RE.findall(line.strip()):
            if word:
                if word.upper() in ("DUP", "DUPLICATE"):
                    continue
                if word.upper() == "COLLEFF":
                    # chemkinFileRead.cpp:345-371: a bimolecular reaction whose
                    # main line is the collision efficiency
                    if cur.kind != "arrhenius":
                        raise ValueError("COLLEFF cannot be used on a third-body or fall-off reaction")
                    if len(cur.fwd) != 2:
                        raise ValueError("The collision reaction should be bimolecular")
                    cur.collision = True
                    continue
                raise ValueError(f"unexpected word {word!r} in {line.strip()!r}")
            up = key.upper()
            v = val.split()
            if up in ("CHEB", "PCHEB", "TCHEB"):
                # ChebyshevPolynomialsRR (ChebyshevPolynomialsRR.cpp:173-236,
                # ChebyshevPolynomialsRR.hpp:85-98, 105-114) evaluates
                # 0.001 log10 of the polynomial sum (the fit is 10 to that
                # power), keeps the transforms of its default 300-2500 K and
                # 0.001-100 atm ranges whatever TCHEB / PCHEB say, and divides
                # its temperature derivative by max(1/Tmax - 1/Tmin, tiny),
                # which is tiny; restating it would give a rate that is not the
                # file's fit, so such reactions are refused
                raise NotImplementedError(
                    f"{up}: the reference's Chebyshev rate (ChebyshevPolynomialsRR) does not "
                    "evaluate the Chebyshev fit (0.001*log10 of the sum, default ranges, "
                    "a 1e-15 divisor in dk/dT); reactions using it are not taken")
            if up in _UNSUPPORTED_AUX:
                raise NotImplementedError(f"rate form {up} is not supported (nor by the "
                                          "reference's reader)")
            if up == "LOW":
                cur.low = (_read_real(v[0]), _read_real(v[1]), _read_real(v[2]))
            elif up == "TROE":
                cur.troe = [_read_real(x) for x in v]
            elif up == "SRI":
                if len(v) not in (3, 5):
                    raise ValueError("SRI takes 3 or 5 parameters")
                cur.sri = [_read_real(x) for x in v]
            elif up == "PLOG":
                # chemkinFileRead.cpp:606-644: PLOG / p[atm] A b E /, not with a third body
                if cur.kind != "arrhenius":
                    raise ValueError("PLOG cannot be used on a third-body or fall-off reaction")
                if len(v) != 4:
                    raise ValueError("PLOG takes a pressure and three Arrhenius parameters")
                if cur.plog is None:
                    cur.plog = []
                cur.plog.append(tuple(_read_real(x) for x in v))
            elif up == "HIGH":
                # chemkinFileRead.cpp:311-344: a (+M) reaction whose main line is k0
                if cur.kind != "falloff":
                    raise ValueError("HIGH needs a pressure-dependent (+M) reaction")
                cur.high = (_read_real(v[0]), _read_real(v[1]), _read_real(v[2]))
            elif up in ("JAN", "FIT1"):
                # chemkinFileRead.cpp:479-529: 9 Janev or 4 power-series coefficients
                # on a reaction without a third body
                if cur.kind != "arrhenius":
                    raise ValueError(f"{up} cannot be used on a third-body or fall-off reaction")
                want = 9 if up == "JAN" else 4
                if len(v) != want:
                    raise ValueError(f"{up} takes {want} coefficients")
                if up == "JAN":
                    cur.janev = [_read_real(x) for x in v]
                else:
                    cur.fit1 = [_read_real(x) for x in v]
            elif up == "LT":
                # chemkinFileRead.cpp:413-440: not on a pressure-dependent reaction
                if cur.kind != "arrhenius":
                    raise ValueError("LT cannot be used on a third-body or fall-off reaction")
                cur.lt = (_read_real(v[0]), _read_real(v[1]))
            elif up == "RLT":
                # chemkinFileRead.cpp:441-478: the reverse rate of a REV reaction in
                # the Landau-Teller form, with REV's A, beta, Ta
                if cur.kind != "arrhenius":
                    raise ValueError("RLT cannot be used on a third-body or fall-off reaction")
                if cur.rev is None:
                    raise ValueError("The keyword RLT must follow the explicit REV parameters")
                cur.rlt = (_read_real(v[0]), _read_real(v[1]))
            elif up == "REV":
                cur.rev = (_read_real(v[0]), _read_real(v[1]), _read_real(v[2]))
            elif up in ("FORD", "RORD"):
                name, order = v[0], _read_real(v[1])
                side = cur.fwd if up == "FORD" else cur.bwd
                if name not in index or index[name] not in [i for i, _ in side]:
                    # chemkinFileRead.cpp:974-1000
                    raise ValueError(f"{up} species {name!r} is not on that side of the reaction")
                d = cur.ford if up == "FORD" else cur.rord
                if d is None:
                    d = {}
                    if up == "FORD":
                        cur.ford = d
                    else:
                        cur.rord = d
                d[index[name]] = order
            elif up == "UNITS":
                kind_u, u = _unit(val, "in UNITS")
                if kind_u == "A":
                    cur.units_A = u
                else:
                    cur.units_E = u
            else:
                if key not in index:
                    raise ValueError(f"unknown efficiency species {key!r}")
                if cur.named_third is not None and index[key] != cur.named_third:
                    raise ValueError(f"the third body of this reaction is "
                                     f"{names[cur.named_third]}, but {key} has an efficiency")
                if cur.eff is None:
                    raise ValueError(f"efficiencies on a reaction without a third body: {line!r}")
                cur.eff[index[key]] = _read_real(val)
    return names, elements, reactions


def parse_thermo(text: str, names: List[str]):
    lines = [l.split("!", 1)[0] if not l.startswith("!") else "" for l in text.splitlines()]
    lines = [l for l in lines if l.strip() != ""]
    glob = None
    for l in lines[:3]:
        nums = l.split()
        if len(nums) == 3:
            try:
                glob = [float(x) for x in nums]
            except ValueError:
                pass
    found = {}
    i = 0
    while i + 3 < len(lines):
        l1 = lines[i]
        if len(l1) >= 80 and l1[79] == "1":
            name = l1[0:18].split()[0]
            if name in names and name not in found:
                tlow = float(l1[45:55])
                thigh = float(l1[55:65])
                tc_txt = l1[65:73].strip()
                tcommon = float(tc_txt) if tc_txt else glob[1]
                elstr = l1[24:44]
                els = []
                for k in range(4):
                    e = elstr[k * 5:k * 5 + 2].strip()
                    c = elstr[k * 5 + 2:k * 5 + 5].strip()
                    if c and int(c) != 0:
                        els.append((e.upper(), int(c)))
                l2, l3, l4 = lines[i + 1], lines[i + 2], lines[i + 3]
                f = lambda l, k: float(l[k * 15:(k + 1) * 15])
                high = [f(l2, 0), f(l2, 1), f(l2, 2), f(l2, 3), f(l2, 4), f(l3, 0), f(l3, 1)]
                low = [f(l3, 2), f(l3, 3), f(l3, 4), f(l4, 0), f(l4, 1), f(l4, 2), f(l4, 3)]
                found[name] = (tlow, tcommon, thigh, els, low, high)
            i += 4
        else:
            i += 1
    missing = [n for n in names if n not in found]
    if missing:
        raise ValueError(f"thermo data missing for {missing}")
    return found


def parse_transport(text: str, names: List[str]):
    out = {}
    for line in text.splitlines():
        line = line.split("!", 1)[0].strip()
        if not line:
            continue
        tok = line.split()
        if tok[0] in names and tok[0] not in out:
            vals = [float(x) for x in tok[1:7]] + [0.0] * (6 - len(tok[1:7]))
            out[tok[0]] = (int(vals[0]), vals[1], vals[2], vals[3], vals[4], vals[5])
    return out


def _embedded(che: str, start_re: str) -> str:
    """A THERMO or TRANSPORT section carried in the mechanism file itself, used
    when no separate file is given (chemkinFileRead.cpp:1700-1718, 1730-1739)."""
    m = re.search(start_re + r"\s+[\s\S]*?\s+END", _strip_comments(che), re.IGNORECASE)
    return m.group(0) if m else ""


def compile_mechanism(che_path: str, thermo_path: Optional[str] = None,
                      transport_path: Optional[str] = None) -> MechTables:
    """Tables from a Chemkin mechanism file and its NASA-7 thermo and transport
    files; without a thermo or transport file, the mechanism file's own
    THERMO / TRANSPORT section is read, as the reference does."""
    with open(che_path) as f:
        che = f.read()
    names, elements, reactions = parse_chemkin(che)
    if thermo_path:
        with open(thermo_path) as f:
            thermo_txt = f.read()
    else:
        thermo_txt = _embedded(che, r"THER(?:MO|)")
    thermo = parse_thermo(thermo_txt, names)
    if transport_path:
        with open(transport_path) as f:
            tran_txt = f.read()
    else:
        tran_txt = _embedded(che, r"TRAN(?:SPORT|)")
    tran = parse_transport(tran_txt, names)
    nsp, nrc = len(names), len(reactions)

    W = np.zeros(nsp)
    Ri = np.zeros(nsp)
    Tr = np.zeros((nsp, 3))
    nasa = np.zeros((nsp, 2, 7))
    el_names = list(elements)
    E = np.zeros((len(el_names), nsp))
    for i, n in enumerate(names):
        tlow, tcommon, thigh, els, low, high = thermo[n]
        w = 0.0
        for e, c in els:
            w += c * ATOMIC_WEIGHTS[e]
            if e not in el_names:
                el_names.append(e)
                E = np.vstack([E, np.zeros((1, nsp))])
            E[el_names.index(e), i] += c
        W[i] = w
        Ri[i] = RU / w
        Tr[i] = (tlow, tcommon, thigh)
        for k in range(7):
            nasa[i, 0, k] = low[k] * Ri[i]
            nasa[i, 1, k] = high[k] * Ri[i]

    rate_type = np.zeros(nrc, np.int32)
    rev = np.zeros(nrc, np.int32)
    arr = np.zeros((nrc, 3))
    arr0 = np.zeros((nrc, 3))
    troe = np.zeros((nrc, 4))
    sri = np.zeros((nrc, 5))
    arr_rev = np.zeros((nrc, 3))
    eff = np.ones((nrc, nsp))
    nf = np.zeros(nrc, np.int32)
    nb = np.zeros(nrc, np.int32)
    fidx = np.zeros((nrc, MAX_SIDE), np.int32)
    bidx = np.zeros((nrc, MAX_SIDE), np.int32)
    fnu = np.zeros((nrc, MAX_SIDE))
    bnu = np.zeros((nrc, MAX_SIDE))
    ford = np.zeros((nrc, MAX_SIDE))
    bord = np.zeros((nrc, MAX_SIDE))
    sum_stoi = np.zeros(nrc)
    plog_rows = []
    activated = np.zeros(nrc, np.int32)
    lt = np.zeros((nrc, 2))
    xcoef = np.zeros((nrc, 9))
    for r, rx in enumerate(reactions):
        if len(rx.fwd) > MAX_SIDE or len(rx.bwd) > MAX_SIDE:
            raise ValueError("too many species on one side")
        fo = [(rx.ford or {}).get(i, nu) for i, nu in rx.fwd]
        bo = [(rx.rord or {}).get(i, nu) for i, nu in rx.bwd]
        # the A factor follows the side's total reaction order, summed in
        # the side's (name-sorted) order (chemkinFileRead.cpp:1365-1371)
        order = 0.0
        for o in fo:
            order += o
        third = rx.kind != "arrhenius"
        Afac, Efac = change_unit(order, rx.units_A, rx.units_E, third)
        if rx.collision:
            if rx.rev is not None:
                raise ValueError("REV cannot be used with a collision rate "
                                 "(chemkinFileRead.cpp:1557-1561)")
            if rx.plog is not None or rx.lt is not None or rx.janev is not None \
                    or rx.fit1 is not None:
                raise ValueError("COLLEFF with another rate form")
            # collisionRR: the Arrhenius line is the efficiency; the collision
            # frequency takes the mean Lennard-Jones diameter of the two
            # reactants as read (angstrom) and their reduced molar mass
            # (chemkinFileRead.cpp:360-371, 1552-1556; collisionRR.cpp:36-42,
            # collisionRR.hpp:94-107)
            (ia, _), (ib, _) = rx.fwd
            for i in (ia, ib):
                if names[i] not in tran:
                    raise ValueError(f"collision reaction needs the transport data of {names[i]}")
            d = 0.0
            d += tran[names[ia]][2]
            d += tran[names[ib]][2]
            d /= 2.0
            WAB = (W[ia] * W[ib]) / (W[ia] + W[ib])
            RAB = RU / WAB
            rate_type[r] = RATE_COLLISION
            arr[r] = (rx.A * Afac, rx.b, rx.E / Efac)
            xcoef[r, :3] = (NA * (d * d), (8.0 * math.pi) * RAB, (2.0 * math.pi) * RAB)
        elif rx.plog is not None:
            if rx.rev is not None:
                raise ValueError("REV cannot be used with a PLOG rate (chemkinFileRead.cpp:1609)")
            # logInterpolationRR::append sorts by pressure after each entry
            # (a stable bubble sort, logInterpolationRR.cpp:37-60); the
            # pressures then become Pa and each entry takes the reaction's
            # unit factors (chemkinFileRead.cpp:1596-1603)
            ent = sorted(rx.plog, key=lambda e: e[0])
            if len(ent) > 1 and ent[-1][0] == ent[-2][0]:
                raise ValueError("PLOG table with its highest pressure twice: the reference's "
                                 "derivative reads past its table there")
            rate_type[r] = RATE_PLOG
            arr[r] = (rx.A * Afac, rx.b, rx.E / Efac)
            plog_rows.append((r, [(pa * PATM, A_ * Afac, b_, E_ / Efac) for pa, A_, b_, E_ in ent]))
        elif rx.rlt is not None and rx.lt is None:
            # the rate type turns Landau-Teller without its LT parameters: the
            # reference aborts there (chemkinFileRead.cpp:1503, a failed cast)
            raise ValueError("RLT on a reaction without LT")
        elif rx.janev is not None or rx.fit1 is not None:
            if rx.rev is not None:
                raise ValueError("REV cannot be used with a Janev or power-series rate")
            # JanevRR: A, beta, Ta from the main line; powerSeriesRR: A and beta
            # only (chemkinFileRead.cpp:1531-1534, 1575-1577)
            if rx.janev is not None:
                rate_type[r] = RATE_JANEV
                arr[r] = (rx.A * Afac, rx.b, rx.E / Efac)
                xcoef[r] = rx.janev
            else:
                rate_type[r] = RATE_POWER_SERIES
                arr[r] = (rx.A * Afac, rx.b, 0.0)
                xcoef[r, :4] = rx.fit1
        elif rx.lt is not None:
            if rx.rev is not None and rx.rlt is None:
                # the reference builds no reverse rate for REV without RLT here
                # (chemkinFileRead.cpp:1507-1512 reads a null one)
                raise ValueError("REV on a Landau-Teller reaction needs RLT")
            rate_type[r] = RATE_LANDAU_TELLER
            arr[r] = (rx.A * Afac, rx.b, rx.E / Efac)
            lt[r] = rx.lt
            if rx.rlt is not None:
                # reverse Landau-Teller B, C beside the REV parameters
                xcoef[r, :2] = rx.rlt
        elif rx.kind == "arrhenius":
            rate_type[r] = RATE_ARRHENIUS
            arr[r] = (rx.A * Afac, rx.b, rx.E / Efac)
        elif rx.kind == "third_body":
            rate_type[r] = RATE_THIRD_BODY
            arr[r] = (1e-3 * rx.A * Afac, rx.b, rx.E / Efac)
            eff[r] = rx.eff
        else:
            if rx.rev is not None:
                raise ValueError("REV cannot be used with a fall-off rate (chemkinFileRead.cpp:1460)")
            if rx.high is not None:
                # chemicallyActicatedBimolecularRR: k0 from the main line, kinf from
                # HIGH, with A factors Afactor and Afactor / 1e-3
                # (chemkinFileRead.cpp:1475-1483)
                if rx.low is not None:
                    raise ValueError("LOW and HIGH on one reaction")
                Ah, bh, Eh = rx.high
                arr0[r] = (rx.A * Afac, rx.b, rx.E / Efac)
                arr[r] = (Ah * (Afac / 1e-3), bh, Eh / Efac)
                activated[r] = 1
            else:
                if rx.low is None:
                    raise ValueError("fall-off reaction without LOW")
                A0, b0, E0 = rx.low
                arr0[r] = (A0 * (1e-3 * Afac), b0, E0 / Efac)
                arr[r] = (rx.A * Afac, rx.b, rx.E / Efac)
            eff[r] = rx.eff
            if rx.sri is not None:
                rate_type[r] = RATE_SRI
                sri[r] = rx.sri if len(rx.sri) == 5 else list(rx.sri) + [1.0, 0.0]
            elif rx.troe is None:
                rate_type[r] = RATE_LINDEMANN
            elif len(rx.troe) == 3:
                rate_type[r] = RATE_TROE3
                troe[r, :3] = rx.troe
            else:
                rate_type[r] = RATE_TROE4
                troe[r, :4] = rx.troe[:4]
        if rx.rev is not None:
            # reversibleReactionWithRevPars: the reverse Arrhenius (or third-body)
            # law with its own A factor from the reverse side's order
            # (chemkinFileRead.cpp:1378-1380, 1387-1421)
            border = 0.0
            for o in bo:
                border += o
            AfR, EfR = change_unit(border, rx.units_A, rx.units_E, third)
            Ar, br, Er = rx.rev
            arr_rev[r] = ((1e-3 * Ar * AfR) if third else (Ar * AfR), br, Er / EfR)
            rev[r] = REVERSIBLE_REV
        else:
            rev[r] = REVERSIBLE if rx.reversible else IRREVERSIBLE
        nf[r], nb[r] = len(rx.fwd), len(rx.bwd)
        s = 0.0
        for k, (i, nu) in enumerate(rx.fwd):
            fidx[r, k], fnu[r, k], ford[r, k] = i, nu, fo[k]
            s -= nu
        for k, (i, nu) in enumerate(rx.bwd):
            bidx[r, k], bnu[r, k], bord[r, k] = i, nu, bo[k]
            s += nu
        sum_stoi[r] = s

    plog_ptr = np.zeros(nrc + 1, np.int32)
    counts = np.zeros(nrc, np.int64)
    for r, ent in plog_rows:
        counts[r] = len(ent)
    plog_ptr[1:] = np.cumsum(counts)
    plog_p = np.zeros(int(plog_ptr[-1]))
    plog_arr = np.zeros((int(plog_ptr[-1]), 3))
    for r, ent in plog_rows:
        for k, (pa, A_, b_, Ta_) in enumerate(ent):
            plog_p[plog_ptr[r] + k] = pa
            plog_arr[plog_ptr[r] + k] = (A_, b_, Ta_)

    geom = np.zeros(nsp, np.int32)
    eps = np.ones(nsp)
    sig = np.ones(nsp)
    dip = np.zeros(nsp)
    pol = np.zeros(nsp)
    zr = np.zeros(nsp)
    for i, n in enumerate(names):
        if n in tran:
            g, e_, s_, d_, p_, z_ = tran[n]
            geom[i], eps[i], sig[i], dip[i], pol[i], zr[i] = g, e_, s_, d_, p_, z_
    return MechTables(names, W, Ri, Tr, nasa, el_names, E, rate_type, rev, arr, arr0, troe,
                      eff, nf, nb, fidx, bidx, fnu, bnu, ford, bord, sum_stoi,
                      geom, eps, sig, dip, pol, zr, sri=sri, arr_rev=arr_rev,
                      plog_ptr=plog_ptr, plog_p=plog_p, plog_arr=plog_arr,
                      activated=activated, lt=lt, xcoef=xcoef)


def element_matrix_mass(m: MechTables) -> np.ndarray:
    """Atoms of each element per kg of each species: E[e, i] / W_i."""
    return m.elem_matrix / m.W[None, :]
