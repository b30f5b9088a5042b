"""ctypes binding of libhurchem_b200.so (include/hurchem_b200.h).

The shared library is built in-tree by openhurricane_b200.build (nvcc,
sm_100a). Loading fails loudly when it is missing: there is no CPU or
library fallback on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# HURCHEM_B200_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("HURCHEM_B200_LIB") or os.path.join(HERE, "libhurchem_b200.so")

HC_MAX_SIDE = 4
HC_CELL_OK = 0
HC_CELL_SKIPPED = 1
HC_CELL_MAXSTEP = 2
HC_CELL_UNDERFLOW = 4
HC_CELL_ITER_LIMIT = 8


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


class HcGateOpts(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("tol_T", "tol_proj", "y_neg", "x_max", "T_min",
                                          "T_max", "tol_spread")]


class HcCounters(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("n_jac", "n_rhs", "n_lu", "n_newton", "n_steps",
                                         "n_attempts")]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


# every symbol include/hurchem_b200.h declares, with its ctypes signature
_VP = C.c_void_p
SIGNATURES = {
    "hc_abi_version": (C.c_int, []),
    "hc_last_error": (C.c_char_p, []),
    "hc_default_opts": (None, [C.POINTER(HcOpts)]),
    "hc_set_tuning": (C.c_int, [_VP, C.c_int, C.c_int]),
    "hc_jit_compile": (C.c_int, [C.POINTER(HcMechDesc), C.c_int, C.POINTER(C.c_int64)]),
    "hc_jit_compile_kernel": (C.c_int, [C.POINTER(HcMechDesc), C.c_int, C.c_int,
                                        C.POINTER(C.c_int64)]),
    "hc_jit_source_kernel": (C.c_int, [C.POINTER(HcMechDesc), C.c_int, C.c_int, C.c_char_p,
                                       C.c_int64, C.POINTER(C.c_int64)]),
    "hc_jit_source": (C.c_int, [C.POINTER(HcMechDesc), C.c_int, C.c_char_p, C.c_int64,
                                C.POINTER(C.c_int64)]),
    "hc_mech_create": (C.c_int, [C.POINTER(HcMechDesc), C.POINTER(_VP)]),
    "hc_mech_destroy": (C.c_int, [_VP]),
    "hc_mech_nsp": (C.c_int, [_VP]),
    "hc_mech_nrc": (C.c_int, [_VP]),
    "hc_integrate": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64] + [_VP] * 5 + [C.c_double] +
                     [_VP] * 4 + [_VP]),
    "hc_integrate_ordered": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64] + [_VP] * 5 +
                             [C.c_double] + [_VP] * 6 + [_VP]),
    "hc_integrate_subset": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64, C.c_int64, _VP] +
                            [_VP] * 5 + [C.c_double] + [_VP] * 5 + [_VP]),
    "hc_integrate_noalloc": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64] + [_VP] * 5 +
                             [C.c_double] + [_VP] * 3 + [_VP]),
    "hc_integrate_host": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64] + [_VP] * 5 +
                          [C.c_double] + [_VP] * 4 + [_VP]),
    "hc_rhs_jacobian": (C.c_int, [_VP, C.c_int64] + [_VP] * 5 + [_VP]),
    "hc_source_terms": (C.c_int, [_VP, C.c_int64] + [_VP] * 5 + [_VP]),
    "hc_properties": (C.c_int, [_VP, C.c_int64] + [_VP] * 8 + [_VP]),
    "hc_source_terms_imp": (C.c_int, [_VP, C.c_int64] + [_VP] * 6 + [_VP]),
    "hc_temperature_from_enthalpy": (C.c_int, [_VP, C.c_int64] + [_VP] * 3 +
                                     [C.c_double, C.c_double] + [_VP] * 3),
    "hc_temperature_from_energy": (C.c_int, [_VP, C.c_int64] + [_VP] * 4 +
                                   [C.c_double, C.c_double] + [_VP] * 3),
    "hc_source_terms_host": (C.c_int, [_VP, C.c_int64] + [_VP] * 5 + [_VP]),
    "hc_properties_host": (C.c_int, [_VP, C.c_int64] + [_VP] * 8 + [_VP]),
    "hc_integrate_aos": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64] + [_VP] * 4 +
                         [C.c_int, _VP, _VP]),
    "hc_integrate_aos_host": (C.c_int, [_VP, C.POINTER(HcOpts), C.c_int64] + [_VP] * 4 +
                              [C.c_int, _VP, _VP]),
    "hc_source_terms_aos": (C.c_int, [_VP, C.c_int64] + [_VP] * 3 + [_VP]),
    "hc_source_terms_aos_async": (C.c_int, [_VP, C.c_int64] + [_VP] * 3 + [_VP]),
    "hc_properties_aos": (C.c_int, [_VP, C.c_int64] + [_VP] * 3 + [_VP]),
    "hc_state_create": (C.c_int, [_VP, C.c_int64, C.POINTER(_VP)]),
    "hc_state_destroy": (C.c_int, [_VP]),
    "hc_state_fields": (C.c_int, [_VP] + [_VP] * 7),
    "hc_upload": (C.c_int, [_VP] + [_VP] * 5 + [_VP]),
    "hc_upload_records": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP]),
    "hc_download": (C.c_int, [_VP] + [_VP] * 6 + [_VP]),
    "hc_download_records": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "hc_state_integrate": (C.c_int, [_VP, C.POINTER(HcOpts), _VP, C.c_double, _VP]),
    "hc_state_source_terms": (C.c_int, [_VP, _VP]),
    "hc_state_properties": (C.c_int, [_VP] + [_VP] * 5 + [_VP]),
    "hc_properties_aos_host": (C.c_int, [_VP, C.c_int64] + [_VP] * 3 + [_VP]),
    "hc_probe_fp64_peak": (C.c_int, [C.c_int, _VP, _VP]),
    "hc_mlp_create": (C.c_int, [C.c_int] * 5 + [C.c_uint64, C.POINTER(_VP)]),
    "hc_mlp_destroy": (C.c_int, [_VP]),
    "hc_mlp_num_params": (C.c_int64, [_VP]),
    "hc_mlp_get_params": (C.c_int, [_VP, _VP]),
    "hc_mlp_set_params": (C.c_int, [_VP, _VP]),
    "hc_mlp_grad": (C.c_int, [_VP, _VP, _VP, C.c_int, _VP, _VP, _VP]),
    "hc_mlp_train_step": (C.c_int, [_VP, _VP, _VP, C.c_int, C.c_float, _VP, C.c_int, _VP]),
    "hc_mlp_forward": (C.c_int, [_VP, _VP, C.c_int64, _VP, _VP]),
    "hc_mlp_check": (C.c_int, [_VP, _VP]),
    "hc_surrogate_features": (C.c_int, [_VP, C.c_int64] + [_VP] * 4 + [C.c_double] + [_VP] * 4),
    "hc_surrogate_gate": (C.c_int, [_VP, C.c_int64] + [_VP] * 10 + [C.c_int] + [_VP] * 6),
    "hc_gemm_bf16_tn": (C.c_int, [_VP, _VP, C.c_int, C.c_int, C.c_int, _VP, C.c_int, _VP, _VP]),
}

_lib: Optional[C.CDLL] = None


NOALLOC_MAX_CELLS = 65536   # HC_NOALLOC_MAX_CELLS


class HcError(RuntimeError):
    pass


def load() -> C.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            raise HcError(f"{LIB_PATH} is missing: run openhurricane_b200.build.build_library() "
                          "(the product has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc: int, what: str) -> int:
    if rc < 0:
        msg = load().hc_last_error().decode(errors="replace")
        raise HcError(f"{what} failed ({rc}): {msg}")
    return rc


def default_opts(**kw) -> HcOpts:
    o = HcOpts()
    load().hc_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class DescArrays:
    """Contiguous numpy copies of the mechanism tables behind an HcMechDesc."""

    def __init__(self, t):
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        self.arrays = dict(
            W=f64(t.W), Trange=f64(t.Trange), nasa=f64(np.asarray(t.nasa).reshape(t.nsp, 14)),
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
        d.nsp, d.nrc = int(t.nsp), int(t.nrc)
        for k, a in self.arrays.items():
            setattr(d, k, a.ctypes.data)
        self.desc = d
