"""ctypes front end of the C restatement (oracle/chem_oracle.c).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "chem_oracle.c")
LIB = os.path.join(HERE, "_build", "libchemoracle.so")
# The reference's Release flags on Linux: -O3 -mavx2 -m64, no -mfma (no contraction).
CFLAGS = ["-std=c11", "-O3", "-mavx2", "-m64", "-fPIC", "-shared", "-ffp-contract=off"]


def build(force: bool = False) -> str:
    if force or not os.path.isfile(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.check_call(["gcc", *CFLAGS, "-o", LIB, SRC, "-lm"])
    return LIB


def _sri(t):
    """SRI parameters [nrc, 5] (zeros for tables without them)."""
    a = getattr(t, "sri", None)
    return np.zeros((t.nrc, 5)) if a is None else a


def _arr_rev(t):
    """Explicit reverse Arrhenius parameters [nrc, 3] (zeros for tables without them)."""
    a = getattr(t, "arr_rev", None)
    return np.zeros((t.nrc, 3)) if a is None else a


def _opt(t, name, shape, dtype):
    """An optional per-reaction table, zeros for tables without it."""
    a = getattr(t, name, None)
    return np.zeros(shape, dtype) if a is None else a


def _plog(t):
    """PLOG tables (ptr [nrc+1], p [n], arr [n, 3]); empty for tables without them.
    The arrays are never empty, so that their addresses are valid."""
    ptr = getattr(t, "plog_ptr", None)
    if ptr is None:
        return np.zeros(t.nrc + 1, np.int32), np.zeros(1), np.zeros((1, 3))
    return (ptr, t.plog_p if len(t.plog_p) else np.zeros(1),
            t.plog_arr if len(t.plog_arr) else np.zeros((1, 3)))


class HcMechDesc(C.Structure):
    _fields_ = [
        ("nsp", C.c_int32), ("nrc", C.c_int32),
        ("W", C.c_void_p), ("Trange", C.c_void_p), ("nasa", C.c_void_p),
        ("rate_type", C.c_void_p), ("reversible", C.c_void_p),
        ("arr", C.c_void_p), ("arr0", C.c_void_p), ("troe", C.c_void_p), ("eff", C.c_void_p),
        ("nf", C.c_void_p), ("nb", C.c_void_p), ("fidx", C.c_void_p), ("bidx", C.c_void_p),
        ("fnu", C.c_void_p), ("bnu", C.c_void_p), ("ford", C.c_void_p), ("bord", C.c_void_p),
        ("geom", C.c_void_p), ("eps_k", C.c_void_p), ("sigma", C.c_void_p),
        ("sri", C.c_void_p), ("arr_rev", C.c_void_p),
        ("plog_ptr", C.c_void_p), ("plog_p", C.c_void_p), ("plog_arr", C.c_void_p),
        ("activated", C.c_void_p), ("lt", C.c_void_p), ("xcoef", C.c_void_p),
    ]


class HcOpts(C.Structure):
    _fields_ = [
        ("maxstep", C.c_int32), ("auto_update_jacobian", C.c_int32),
        ("step_to_update_jac", C.c_int32), ("reactor", C.c_int32),
        ("atol", C.c_double), ("rtol", C.c_double), ("safescale", C.c_double),
        ("minscale", C.c_double), ("maxscale", C.c_double), ("alphainc", C.c_double),
        ("atol_increment", C.c_double), ("rtol_increment", C.c_double),
        ("T_threshold", C.c_double), ("T_alpha", C.c_double), ("T_beta", C.c_double),
        ("dt_max", C.c_double), ("max_newton_total", C.c_int64),
    ]


class HcCounters(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("n_jac", "n_rhs", "n_lu", "n_newton", "n_steps",
                                         "n_attempts")]


def default_opts(**kw) -> HcOpts:
    o = HcOpts(maxstep=10000, auto_update_jacobian=0, step_to_update_jac=10, reactor=0,
               atol=1e-15, rtol=1e-4, safescale=0.8, minscale=0.25, maxscale=2.0,
               alphainc=0.25, atol_increment=1e-7, rtol_increment=1e-3, T_threshold=200.0,
               T_alpha=0.2, T_beta=0.25, dt_max=1e15, max_newton_total=0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class MechDesc:
    """Keeps the numpy arrays alive behind an HcMechDesc."""

    def __init__(self, t):
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        self.arrays = dict(
            W=f64(t.W), Trange=f64(t.Trange), nasa=f64(t.nasa.reshape(t.nsp, 14)),
            rate_type=i32(t.rate_type), reversible=i32(t.reversible), arr=f64(t.arr),
            arr0=f64(t.arr0), troe=f64(t.troe), eff=f64(t.eff), nf=i32(t.nf), nb=i32(t.nb),
            fidx=i32(t.fidx), bidx=i32(t.bidx), fnu=f64(t.fnu), bnu=f64(t.bnu),
            ford=f64(t.ford), bord=f64(t.bord), geom=i32(t.geom), eps_k=f64(t.eps_k),
            sigma=f64(t.sigma), sri=f64(_sri(t)), arr_rev=f64(_arr_rev(t)),
            plog_ptr=i32(_plog(t)[0]), plog_p=f64(_plog(t)[1]), plog_arr=f64(_plog(t)[2]),
            activated=i32(_opt(t, "activated", (t.nrc,), np.int32)),
            lt=f64(_opt(t, "lt", (t.nrc, 2), np.float64)),
            xcoef=f64(_opt(t, "xcoef", (t.nrc, 9), np.float64)))
        d = HcMechDesc()
        d.nsp, d.nrc = t.nsp, t.nrc
        for k, a in self.arrays.items():
            setattr(d, k, a.ctypes.data)
        self.desc = d
        self.nsp, self.nrc = t.nsp, t.nrc


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.oracle_integrate.restype = C.c_int
        _lib.oracle_integrate.argtypes = [C.POINTER(HcMechDesc), C.POINTER(HcOpts), C.c_int64] + \
            [C.c_void_p] * 5 + [C.c_double] + [C.c_void_p] * 4
        _lib.oracle_rhs_jac.argtypes = [C.POINTER(HcMechDesc), C.c_int64] + [C.c_void_p] * 5
        _lib.oracle_thermo.argtypes = [C.POINTER(HcMechDesc), C.c_double, C.c_void_p]
        _lib.oracle_rates.argtypes = [C.POINTER(HcMechDesc), C.c_double, C.c_double, C.c_void_p,
                                      C.c_void_p]
    return _lib


def _p(a):
    return a.ctypes.data


def _threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def integrate(md: MechDesc, T, p, rho, Y, dt, subdt=None, dt_factor=1.0,
              opts: Optional[HcOpts] = None, threads: Optional[int] = None) -> Dict[str, np.ndarray]:
    """Integrate every cell (the C restatement is re-entrant; cells are split
    into contiguous slices over `threads` host threads, ctypes releasing the
    GIL during each call)."""
    n = int(np.asarray(T).shape[0])
    T = np.array(T, dtype=np.float64, copy=True)
    p = np.ascontiguousarray(np.broadcast_to(np.asarray(p, np.float64), (n,)))
    rho = np.array(np.broadcast_to(np.asarray(rho, np.float64), (n,)), copy=True)
    Y = np.array(Y, dtype=np.float64, copy=True, order="C")
    dt = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (n,)))
    sub = np.array(dt if subdt is None else np.broadcast_to(np.asarray(subdt, np.float64), (n,)),
                   dtype=np.float64, copy=True)
    c = np.zeros_like(Y)
    st = np.zeros(n, np.int32)
    o = opts or default_opts()
    nth = max(1, min(threads or _threads(), n))
    bounds = np.linspace(0, n, nth + 1).astype(np.int64)
    L = lib()

    def one(k):
        a, b = int(bounds[k]), int(bounds[k + 1])
        if b <= a:
            return 0, HcCounters()
        Ts, ps, rs = T[a:b].copy(), p[a:b].copy(), rho[a:b].copy()
        Ys, ds, ss = np.ascontiguousarray(Y[:, a:b]), dt[a:b].copy(), sub[a:b].copy()
        cs, sts = np.zeros_like(Ys), np.zeros(b - a, np.int32)
        cnt = HcCounters()
        rc = L.oracle_integrate(C.byref(md.desc), C.byref(o), b - a, _p(Ts), _p(ps), _p(rs),
                                _p(Ys), _p(ds), dt_factor, _p(ss), _p(cs), _p(sts),
                                C.addressof(cnt))
        T[a:b], rho[a:b], Y[:, a:b], sub[a:b], c[:, a:b], st[a:b] = Ts, rs, Ys, ss, cs, sts
        return rc, cnt

    if nth == 1:
        parts = [one(0)]
    else:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=nth) as ex:
            parts = list(ex.map(one, range(nth)))
    rc = sum(r for r, _ in parts)
    counters = {k: int(sum(getattr(cn, k) for _, cn in parts)) for k, _ in HcCounters._fields_}
    return {"T": T, "rho": rho, "Y": Y, "c": c, "subdt": sub, "status": st, "rc": rc,
            "counters": counters}


def rhs_jac(md: MechDesc, c, T, p=None):
    """DyDt and the Jacobian at states (c [nsp, ns], T [ns]) and pressures p
    ([ns] or a scalar; one atmosphere when None -- only pressure-dependent rate
    tables read it)."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    ns = T.shape[0]
    n = md.nsp + 1
    dydt = np.zeros((ns, n))
    J = np.zeros((ns, n, n))
    pp = None if p is None else np.ascontiguousarray(np.broadcast_to(np.asarray(p, np.float64), (ns,)))
    lib().oracle_rhs_jac(C.byref(md.desc), ns, _p(c), _p(T), None if pp is None else _p(pp),
                         _p(dydt), _p(J))
    return dydt, J


def thermo(md: MechDesc, T: float) -> np.ndarray:
    out = np.zeros((md.nsp, 7))
    lib().oracle_thermo(C.byref(md.desc), float(T), _p(out))
    return out


def rates(md: MechDesc, T: float, c, p: float = 101325.0) -> np.ndarray:
    c = np.ascontiguousarray(c, dtype=np.float64)
    out = np.zeros((md.nrc, 3))
    lib().oracle_rates(C.byref(md.desc), float(p), float(T), _p(c), _p(out))
    return out
