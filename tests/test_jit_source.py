"""The mechanism-specialised kernel's generated source (hc_jit_source) is
produced without a GPU and compiles for sm_100a."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _source(tables, block=64):
    from openhurricane_b200 import _capi
    lib = _capi.load()
    d = _capi.DescArrays(tables)
    n = C.c_int64(0)
    _capi.check(lib.hc_jit_source(C.byref(d.desc), block, None, 0, C.byref(n)), "hc_jit_source")
    buf = C.create_string_buffer(n.value + 1)
    _capi.check(lib.hc_jit_source(C.byref(d.desc), block, buf, n.value + 1, C.byref(n)),
                "hc_jit_source")
    return buf.value.decode()


def test_source_has_literals_and_entry(small):
    src = _source(small["tables"])
    assert 'extern "C" __global__' in src and "hc_jit_t1" in src
    assert "N = 10" in src and "B = 64" in src
    # every reaction is unrolled
    assert src.count("// reaction ") == small["tables"].nrc


def test_large_mechanism_has_no_generated_kernel(large):
    from openhurricane_b200 import _capi
    lib = _capi.load()
    d = _capi.DescArrays(large["tables"])
    n = C.c_int64(0)
    assert lib.hc_jit_source(C.byref(d.desc), 64, None, 0, C.byref(n)) == -3


def test_generated_source_compiles_for_sm100a(small, tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    f = tmp_path / "gen.cu"
    f.write_text(_source(small["tables"], 64))
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
                        "-I", os.path.join(ROOT, "openhurricane_b200", "csrc"), "-c", str(f),
                        "-o", str(tmp_path / "gen.o")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]


def test_nvrtc_compiles_generated_kernel(small):
    """The library's own NVRTC path (no GPU needed to compile)."""
    from openhurricane_b200 import _capi
    lib = _capi.load()
    d = _capi.DescArrays(small["tables"])
    n = C.c_int64(0)
    rc = lib.hc_jit_compile(C.byref(d.desc), 64, C.byref(n))
    if rc == -3 and b"NVRTC" in lib.hc_last_error():
        pytest.skip("NVRTC not available here")
    _capi.check(rc, "hc_jit_compile")
    assert n.value > 10000
