"""The C++ host interface (include/hurchem_b200.hpp) compiles and links
against the library without a GPU; on a GPU its solveUpdate, per-cell solve
and calculateSourceTerms agree with the oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "solve_cells.cpp")
LIBDIR = os.path.join(ROOT, "openhurricane_b200")


def _compile(tmp_path):
    exe = str(tmp_path / "solve_cells")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), SRC,
           "-o", exe, "-L", LIBDIR, "-lhurchem_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_host_compiles_and_links(tmp_path):
    if not os.path.isfile(os.path.join(LIBDIR, "libhurchem_b200.so")):
        pytest.fail("library not built")
    _compile(tmp_path)


def _write_input(path, t, T, p, rho, Y, dt, atol, rtol):
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32).tobytes()
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64).tobytes()
    n = T.shape[0]
    with open(path, "wb") as f:
        f.write(np.array([t.nsp, t.nrc], np.int32).tobytes())
        f.write(np.array([n], np.int64).tobytes())
        f.write(f64(t.W) + f64(t.Trange) + f64(t.nasa.reshape(t.nsp, 14)))
        f.write(i32(t.rate_type) + i32(t.reversible))
        f.write(f64(t.arr) + f64(t.arr0) + f64(t.troe) + f64(t.eff))
        f.write(i32(t.nf) + i32(t.nb) + i32(t.fidx) + i32(t.bidx))
        f.write(f64(t.fnu) + f64(t.bnu) + f64(t.ford) + f64(t.bord))
        f.write(i32(t.geom) + f64(t.eps_k) + f64(t.sigma))
        f.write(f64(T) + f64(p) + f64(rho) + f64(Y) + f64(dt) + f64([atol, rtol]))


@pytest.mark.gpu
def test_cpp_host_matches_oracle(tmp_path, small):
    from openhurricane_b200 import synth
    from oracle import port
    t = small["tables"]
    c = synth.dirichlet_cells(t.nsp, 64, seed=91)
    rho = synth.mixture_density(t.W, c)
    dt = np.full(64, 1e-6)
    exe = _compile(tmp_path)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write_input(fin, t, c.T, c.p, rho, c.Y, dt, 1e-15, 1e-6)
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(fout, dtype=np.float64)
    n, ns = 64, t.nsp
    T, rho_o = out[:n], out[n:2 * n]
    Y = out[2 * n:2 * n + ns * n].reshape(ns, n)
    Ri = out[2 * n + ns * n:2 * n + 2 * ns * n].reshape(ns, n)
    T0 = out[-1]
    o = port.integrate(port.MechDesc(t), c.T, c.p, rho, c.Y, 1e-6,
                       opts=port.default_opts(atol=1e-15, rtol=1e-6))
    assert np.max(np.abs(T - o["T"]) / o["T"]) <= 1e-6
    assert np.max(np.abs(Y - o["Y"]) - 1e-5 * np.abs(o["Y"]) - 1e-12) <= 0
    assert abs(T0 - o["T"][0]) / o["T"][0] <= 1e-6
    # source terms at the new state against the oracle's right-hand side
    cc = rho_o[None, :] * Y / t.W[:, None]
    f, _ = port.rhs_jac(port.MechDesc(t), cc, T)
    ref = f[:, :ns].T * t.W[:, None]
    # near equilibrium the net rates are differences of large forward and
    # reverse rates: compare against the cell's largest term with 1e-9
    sc = np.abs(ref).max(axis=0, keepdims=True) + 1e-300
    assert (np.abs(Ri - ref) / sc).max() < 1e-9
