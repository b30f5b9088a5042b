"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(hc_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("hc_mech_create", "hc_integrate", "hc_integrate_host", "hc_source_terms",
                 "hc_properties", "hc_rhs_jacobian", "hc_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from openhurricane_b200 import _capi
    if not os.path.isfile(_capi.LIB_PATH):
        pytest.fail("libhurchem_b200.so not built: python -m openhurricane_b200.build")
    lib = _capi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in _capi.SIGNATURES, name
    assert lib.hc_abi_version() == 2


def test_default_opts_match_reference_defaults():
    from openhurricane_b200 import _capi
    o = _capi.default_opts()
    assert (o.maxstep, o.rtol, o.atol, o.safescale, o.minscale, o.maxscale, o.alphainc) == \
        (10000, 1e-4, 1e-15, 0.8, 0.25, 2.0, 0.25)
    assert (o.atol_increment, o.rtol_increment, o.step_to_update_jac) == (1e-7, 1e-3, 10)
    assert (o.T_threshold, o.T_alpha, o.T_beta) == (200.0, 0.2, 0.25)


def test_invalid_arguments_fail_loudly_without_gpu():
    from openhurricane_b200 import _capi
    lib = _capi.load()
    h = C.c_void_p()
    assert lib.hc_mech_create(None, C.byref(h)) == -1
    assert b"null" in lib.hc_last_error()
    assert lib.hc_set_tuning(None, 0, 64) == -1


def test_mechanism_checks_of_the_extended_rate_forms_without_gpu(ext):
    """SRI and explicit reverse (REV) reactions: the generated thread-per-cell
    kernel refuses them, and inconsistent tables are rejected before any
    device work (hc_jit_source runs the mechanism checks on the host)."""
    from openhurricane_b200 import _capi
    lib = _capi.load()
    n = C.c_int64()
    a = _capi.DescArrays(ext["tables"])
    assert lib.hc_jit_source(C.byref(a.desc), 64, None, 0, C.byref(n)) == -3
    assert b"SRI" in lib.hc_last_error()

    def bad(mutate, msg):
        import copy
        b = _capi.DescArrays(copy.deepcopy(ext["tables"]))    # the arrays may alias the tables
        mutate(b)
        assert lib.hc_jit_source(C.byref(b.desc), 64, None, 0, C.byref(n)) == -1
        assert msg in lib.hc_last_error()

    bad(lambda b: setattr(b.desc, "sri", None), b"SRI reaction without")
    bad(lambda b: setattr(b.desc, "arr_rev", None), b"REV reaction without")

    def rev_on_falloff(b):
        b.arrays["reversible"][b.arrays["rate_type"] == 5] = 2
    bad(rev_on_falloff, b"fall-off")

    def bad_code(b):
        b.arrays["reversible"][0] = 3
    bad(bad_code, b"reversibility")


def test_mechanism_checks_of_the_fitted_rate_forms_without_gpu(fitted):
    """Janev, power-series, reverse Landau-Teller and collision reactions: the
    generated thread-per-cell kernel refuses them; their coefficient table,
    explicit reverse parameters where they cannot be, and unknown rate codes
    are rejected on the host."""
    import copy
    from openhurricane_b200 import _capi
    lib = _capi.load()
    n = C.c_int64()
    a = _capi.DescArrays(fitted["tables"])
    assert lib.hc_jit_source(C.byref(a.desc), 64, None, 0, C.byref(n)) == -3
    assert b"collision" in lib.hc_last_error()

    def bad(mutate, msg):
        b = _capi.DescArrays(copy.deepcopy(fitted["tables"]))
        mutate(b)
        assert lib.hc_jit_source(C.byref(b.desc), 64, None, 0, C.byref(n)) == -1
        assert msg in lib.hc_last_error()

    bad(lambda b: setattr(b.desc, "xcoef", None), b"without coefficients")

    def rev_on_collision(b):
        b.arrays["reversible"][b.arrays["rate_type"] == 10] = 2
    bad(rev_on_collision, b"explicit reverse parameters on a Janev / power-series / collision")

    def unknown_code(b):
        b.arrays["rate_type"][b.arrays["rate_type"] == 10] = 11
    bad(unknown_code, b"unknown rate type")


def test_state_api_rejects_null_handles_without_gpu():
    from openhurricane_b200 import _capi
    lib = _capi.load()
    st = C.c_void_p()
    assert lib.hc_state_create(None, 16, C.byref(st)) == -1
    assert b"null mechanism" in lib.hc_last_error()
    assert lib.hc_upload(None, None, None, None, None, None, None) == -1
    assert lib.hc_download(None, None, None, None, None, None, None, None) == -1
    assert lib.hc_state_integrate(None, C.byref(_capi.default_opts()), None, 1.0, None) == -1
    assert lib.hc_state_destroy(None) == 0
