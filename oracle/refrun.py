"""Run the reference's own CPU chemistry path (oracle/_ref/hurchem_ref).

TEST INFRASTRUCTURE: used only by tests/, the fixture script under
tests/golden/ and the CPU-baseline leg of bench.py, as the checker and the
timed CPU baseline. Nothing in the product imports this module.

The binary is built by oracle/Makefile.ref from the reference sources; see
oracle/ref_driver.cpp for the modes and binary formats. The reference's
chemistry object is not thread-safe (chemistrySource.hpp:80-84 keeps mutable
scratch and the reaction list shares one G0 array), so parallel runs use one
process per core on contiguous cell slices, as the reference's MPI ranks do.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "hurchem_ref")


def available() -> bool:
    return os.path.isfile(REF_BIN) and os.access(REF_BIN, os.X_OK)


def write_case(path: str, che: str, thermo: str, tran: str, opts: Optional[Dict] = None) -> None:
    """Case file for the driver: the mixture files and the chemistry-source
    solver options, in the reference's XML controller format (merged over the
    built-in chemSolvers configuration by the driver). The property mode needs
    a viscous flow model (flowModel="laminarFlow"): with the inviscid EulerFlow
    the reference does not read transport data."""
    o = dict(ODEsSolver="ImplicitEuler", maxstep=10000, atol=1e-11, rtol=1e-4,
             safescale=0.8, minscale=0.25, maxScale=2.0, alphainc=0.25,
             autoUpdateJacobian="off", stepToUpdateJac=10, ATolIncrement=1e-7,
             RTolIncrement=1e-3, TemperatureThreshold=200.0, TemperatureAlpha=0.2,
             TemperatureBeta=0.25, chemicalMaxStep=1e10, reactor="constPressure",
             flowModel="EulerFlow")
    if opts:
        o.update(opts)
    xml = f"""<?xml version="1.0" encoding="UTF-8" standalone="no"?>
<Config>
  <flow>
    <flowModel>{o['flowModel']}</flowModel>
    <mixture>
      <equationOfState>perfectGas</equationOfState>
      <chemical>reaction</chemical>
      <thermo><type>JANAF</type></thermo>
      <transport><type>kinetic</type></transport>
      <mixtureFiles>
        <chemFile>{os.path.abspath(che)}</chemFile>
        <thermoFile>{os.path.abspath(thermo)}</thermoFile>
        <tansportFile>{os.path.abspath(tran)}</tansportFile>
      </mixtureFiles>
      <reactions>
        <chemistrySource>
          <solver>
            <ODEsSolver>{o['ODEsSolver']}</ODEsSolver>
            <maxstep>{o['maxstep']}</maxstep>
            <atol>{o['atol']!r}</atol>
            <rtol>{o['rtol']!r}</rtol>
            <safescale>{o['safescale']!r}</safescale>
            <minscale>{o['minscale']!r}</minscale>
            <maxScale>{o['maxScale']!r}</maxScale>
            <alphainc>{o['alphainc']!r}</alphainc>
            <ImplicitEuler>
              <autoUpdateJacobian>{o['autoUpdateJacobian']}</autoUpdateJacobian>
              <stepToUpdateJac>{o['stepToUpdateJac']}</stepToUpdateJac>
              <ATolIncrement>{o['ATolIncrement']!r}</ATolIncrement>
              <RTolIncrement>{o['RTolIncrement']!r}</RTolIncrement>
            </ImplicitEuler>
          </solver>
          <chemistrySource>chemistryODEs</chemistrySource>
          <chemicalMaxStep>{o['chemicalMaxStep']!r}</chemicalMaxStep>
          <solveOptions>
            <TemperatureThreshold>{o['TemperatureThreshold']!r}</TemperatureThreshold>
            <TemperatureAlpha>{o['TemperatureAlpha']!r}</TemperatureAlpha>
            <TemperatureBeta>{o['TemperatureBeta']!r}</TemperatureBeta>
          </solveOptions>
        </chemistrySource>
      </reactions>
    </mixture>
  </flow>
  <chemSolvers>
    <type>{o['reactor']}</type>
  </chemSolvers>
</Config>
"""
    with open(path, "w") as f:
        f.write(xml)


def write_cells(path: str, T, p, rho, dt, subdt0, Y) -> None:
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    nsp, n = Y.shape
    with open(path, "wb") as f:
        np.array([nsp, n], dtype=np.int64).tofile(f)
        for a in (T, p, rho, dt, subdt0):
            np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64), (n,))).tofile(f)
        Y.tofile(f)


def read_result(path: str) -> Dict[str, np.ndarray]:
    raw = np.fromfile(path, dtype=np.int64, count=2)
    nsp, n = int(raw[0]), int(raw[1])
    d = np.fromfile(path, dtype=np.float64, offset=16)
    out = {}
    off = 0
    for k in ("T", "p", "rho", "subdt", "status"):
        out[k] = d[off:off + n]
        off += n
    out["Y"] = d[off:off + nsp * n].reshape(nsp, n)
    off += nsp * n
    out["c"] = d[off:off + nsp * n].reshape(nsp, n)
    return out


def _run(case: str, env: Dict[str, str], cwd: str) -> str:
    e = dict(os.environ)
    e.update(env)
    r = subprocess.run([REF_BIN, "-i", case], env=e, cwd=cwd, capture_output=True, text=True,
                       timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(f"reference driver failed rc={r.returncode}: {r.stderr[-2000:]}"
                           f"{r.stdout[-2000:]}")
    return r.stderr


def integrate(case: str, T, p, rho, dt, subdt0, Y, procs: int = 1,
              workdir: Optional[str] = None) -> Dict[str, np.ndarray]:
    """Integrate every cell with the reference; returns the result arrays and
    'seconds' = the max over processes of the integration loop's wall time."""
    tmp = workdir or tempfile.mkdtemp(prefix="hcref_")
    cells = os.path.join(tmp, "cells.bin")
    write_cells(cells, T, p, rho, dt, subdt0, Y)
    n = np.asarray(Y).shape[1]
    procs = max(1, min(procs, n))
    bounds = np.linspace(0, n, procs + 1).astype(int)

    def one(k):
        out = os.path.join(tmp, f"res_{k}.bin")
        err = _run(case, {"HC_MODE": "integrate", "HC_IN": cells, "HC_OUT": out,
                          "HC_BEGIN": str(bounds[k]), "HC_END": str(bounds[k + 1]),
                          "OMP_NUM_THREADS": "1"}, tmp)
        secs = 0.0
        for line in err.splitlines():
            if line.startswith("HC_INTEGRATE_SECONDS"):
                secs = float(line.split()[1])
        return read_result(out), secs

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=procs) as ex:
        parts = list(ex.map(one, range(procs)))
    wall = time.perf_counter() - t0
    res = {}
    for k in ("T", "p", "rho", "subdt", "status"):
        res[k] = np.concatenate([pr[0][k] for pr in parts])
    for k in ("Y", "c"):
        res[k] = np.concatenate([pr[0][k] for pr in parts], axis=1)
    res["seconds"] = max(pr[1] for pr in parts)
    res["wall"] = wall
    res["procs"] = procs
    return res


def kat(case: str, p, T, c, workdir: Optional[str] = None) -> Dict[str, np.ndarray]:
    """Evaluate DyDt, the analytic Jacobian, species thermo and reaction rate
    constants at the given states with the reference."""
    tmp = workdir or tempfile.mkdtemp(prefix="hckat_")
    c = np.ascontiguousarray(c, dtype=np.float64)
    nsp, n = c.shape
    path = os.path.join(tmp, "states.bin")
    with open(path, "wb") as f:
        np.array([nsp, n], dtype=np.int64).tofile(f)
        np.asarray(p, np.float64).tofile(f)
        np.asarray(T, np.float64).tofile(f)
        c.tofile(f)
    out = os.path.join(tmp, "kat.bin")
    _run(case, {"HC_MODE": "kat", "HC_IN": path, "HC_OUT": out}, tmp)
    hdr = np.fromfile(out, dtype=np.int64, count=3)
    nsp, nrc, n = (int(x) for x in hdr)
    d = np.fromfile(out, dtype=np.float64, offset=24)
    neq = nsp + 1
    per = neq + neq * neq + 7 * nsp + 3 * nrc
    d = d.reshape(n, per)
    o = 0
    res = {"dydt": d[:, o:o + neq]}
    o += neq
    res["J"] = d[:, o:o + neq * neq].reshape(n, neq, neq)
    o += neq * neq
    th = d[:, o:o + 7 * nsp].reshape(n, nsp, 7)
    o += 7 * nsp
    for k, name in enumerate(("cp0", "ha0", "s0", "g0", "G0", "DG0DT", "Dcp_pDT")):
        res[name] = th[:, :, k]
    rr = d[:, o:o + 3 * nrc].reshape(n, nrc, 3)
    res["kf"], res["Kc"], res["kr"] = rr[:, :, 0], rr[:, :, 1], rr[:, :, 2]
    return res


def props(case: str, T, p, rho, Y, workdir: Optional[str] = None) -> Dict[str, np.ndarray]:
    tmp = workdir or tempfile.mkdtemp(prefix="hcprop_")
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    nsp, n = Y.shape
    cells = os.path.join(tmp, "cells.bin")
    write_cells(cells, T, p, rho, 0.0, 0.0, Y)
    out = os.path.join(tmp, "props.bin")
    err = _run(case, {"HC_MODE": "props", "HC_IN": cells, "HC_OUT": out}, tmp)
    secs = 0.0
    for line in err.splitlines():
        if line.startswith("HC_PROPS_SECONDS"):
            secs = float(line.split()[1])
    d = np.fromfile(out, dtype=np.float64, offset=16).reshape(n, 2 * nsp + 3)
    return {"ha": d[:, :nsp].T.copy(), "cp": d[:, nsp].copy(), "mu": d[:, nsp + 1].copy(),
            "kappa": d[:, nsp + 2].copy(), "D": d[:, nsp + 3:].T.copy(), "seconds": secs}


def srcimp(case: str, T, p, rho, Y, workdir: Optional[str] = None) -> Dict[str, np.ndarray]:
    """The reference's point-implicit source terms at the given states:
    Ri [nsp, n] and the diagonal source Jacobian diag [nsp-1, n]
    (chemistrySource::calculateSourceTermsImp with withoutLastSpec = true)."""
    tmp = workdir or tempfile.mkdtemp(prefix="hcsrc_")
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    nsp, n = Y.shape
    cells = os.path.join(tmp, "cells_src.bin")
    write_cells(cells, T, p, rho, 0.0, 0.0, Y)
    out = os.path.join(tmp, "srcimp.bin")
    _run(case, {"HC_MODE": "srcimp", "HC_IN": cells, "HC_OUT": out}, tmp)
    d = np.fromfile(out, dtype=np.float64, offset=16).reshape(n, 2 * nsp - 1)
    return {"Ri": d[:, :nsp].T.copy(), "diag": d[:, nsp:].T.copy()}


def tha(case: str, ha, p, T0, Y, workdir: Optional[str] = None) -> Dict[str, np.ndarray]:
    """The reference's temperature from mixture enthalpy at constant p
    (thermoList::THa_p) for each cell, starting from T0; returns T and iFlag."""
    tmp = workdir or tempfile.mkdtemp(prefix="hctha_")
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    nsp, n = Y.shape
    cells = os.path.join(tmp, "cells_tha.bin")
    # the cells format carries ha in the dt column and T0 in the subDt0 column
    write_cells(cells, np.asarray(T0, np.float64), p, np.ones(n), ha, T0, Y)
    out = os.path.join(tmp, "tha.bin")
    _run(case, {"HC_MODE": "tha", "HC_IN": cells, "HC_OUT": out}, tmp)
    d = np.fromfile(out, dtype=np.float64, offset=8).reshape(n, 2)
    return {"T": d[:, 0].copy(), "iflag": d[:, 1].astype(np.int32)}


def tea(case: str, ea, rho, T0, Y, workdir: Optional[str] = None) -> Dict[str, np.ndarray]:
    """The reference's temperature from mixture internal energy at constant
    density (thermoList::TEa_rho) for each cell, starting from T0; returns T
    and iFlag."""
    tmp = workdir or tempfile.mkdtemp(prefix="hctea_")
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    nsp, n = Y.shape
    cells = os.path.join(tmp, "cells_tea.bin")
    # the cells format carries ea in the dt column and T0 in the subDt0 column
    write_cells(cells, np.asarray(T0, np.float64), np.full(n, 101325.0), rho, ea, T0, Y)
    out = os.path.join(tmp, "tea.bin")
    _run(case, {"HC_MODE": "tea", "HC_IN": cells, "HC_OUT": out}, tmp)
    d = np.fromfile(out, dtype=np.float64, offset=8).reshape(n, 2)
    return {"T": d[:, 0].copy(), "iflag": d[:, 1].astype(np.int32)}
