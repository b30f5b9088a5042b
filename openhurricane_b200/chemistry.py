"""Host-side mirror of the reference's chemistry-source interface.

`ChemistrySource` keeps the call signatures the reference's flow solver uses
(chemistrySource.hpp:576-662) over device-resident structure-of-arrays fields:

    solve(dt, dtFactor) -> min sub-step; fills Ri   (chemistrySource.cpp:1494-1556)
    solveUpdate(dt, dtFactor): Y, T updated in place (chemistrySource.cpp:1558-1609)
    calculateSourceTerms(): Ri = omega_i W_i        (chemistrySource.cpp:1370-1406)
    Ri(i): species i's source term [kg/m^3/s]

Every call goes through the C ABI of libhurchem_b200.so (include/hurchem_b200.h);
torch is used only to hold device memory and to provide the stream.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, Optional

import numpy as np
import torch

from . import _capi
from .mechanism import MechTables, compile_mechanism


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _f64(t: torch.Tensor, name: str) -> torch.Tensor:
    if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float64 CUDA tensor")
    return t


class Mechanism:
    """A mechanism uploaded to the GPU (hc_mech_create)."""

    def __init__(self, tables: MechTables):
        self.tables = tables
        lib = _capi.load()
        self._desc = _capi.DescArrays(tables)
        h = C.c_void_p()
        _capi.check(lib.hc_mech_create(C.byref(self._desc.desc), C.byref(h)), "hc_mech_create")
        self.handle = h
        self.nsp = tables.nsp
        self.nrc = tables.nrc
        self.W = torch.tensor(tables.W, dtype=torch.float64)

    @classmethod
    def from_chemkin(cls, che: str, thermo: str, transport: str) -> "Mechanism":
        return cls(compile_mechanism(che, thermo, transport))

    def set_tuning(self, kernel: int = 0, block: int = 64):
        """kernel: 0 automatic (warp per cell where it applies, else the cell group),
        1 table-driven thread per cell, 2 cell group,
        3 generated thread per cell, 4 compact thread per cell, 5 generated direct-assembly
        thread per cell, 6 warp per cell, 7 segment per cell (see hc_set_tuning)."""
        _capi.check(_capi.load().hc_set_tuning(self.handle, int(kernel), int(block)),
                    "hc_set_tuning")

    def close(self):
        if getattr(self, "handle", None):
            _capi.load().hc_mech_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rhs_jacobian(self, c: torch.Tensor, T: torch.Tensor, p: torch.Tensor, jac: bool = True,
                     stream=None):
        """f = d[c, T]/dt and the analytic Jacobian at states (c: [nsp, n])."""
        n = T.shape[0]
        n1 = self.nsp + 1
        dydt = torch.empty((n, n1), dtype=torch.float64, device=T.device)
        J = torch.empty((n, n1, n1), dtype=torch.float64, device=T.device) if jac else None
        rc = _capi.load().hc_rhs_jacobian(self.handle, n, _ptr(_f64(c, "c")), _ptr(_f64(T, "T")),
                                          _ptr(_f64(p, "p")), _ptr(dydt), _ptr(J), _stream(stream))
        _capi.check(rc, "hc_rhs_jacobian")
        return dydt, J

    def source_terms(self, T, p, rho, Y, stream=None) -> torch.Tensor:
        Ri = torch.empty_like(Y)
        rc = _capi.load().hc_source_terms(self.handle, T.shape[0], _ptr(_f64(T, "T")),
                                          _ptr(_f64(p, "p")), _ptr(_f64(rho, "rho")),
                                          _ptr(_f64(Y, "Y")), _ptr(Ri), _stream(stream))
        _capi.check(rc, "hc_source_terms")
        return Ri

    def source_terms_aos(self, YiRhoT, p=None, stream=None) -> torch.Tensor:
        """RRi [n, nsp] from records [n, nsp+2] = [Y_0..Y_{nsp-1}, rho, T] (the
        reference's CUDA source-term buffers); p from the ideal-gas law when None."""
        n = YiRhoT.shape[0]
        if YiRhoT.dim() != 2 or YiRhoT.shape[1] != self.nsp + 2:
            raise ValueError("records must be [n, nsp + 2]")
        RRi = torch.empty((n, self.nsp), dtype=torch.float64, device=YiRhoT.device)
        rc = _capi.load().hc_source_terms_aos(self.handle, n, _ptr(_f64(YiRhoT, "YiRhoT")),
                                              _ptr(None if p is None else _f64(p, "p")),
                                              _ptr(RRi), _stream(stream))
        _capi.check(rc, "hc_source_terms_aos")
        return RRi

    def integrate_aos(self, TYiRho, dt, subdt, p=None, return_ci: bool = True, opts=None,
                      stream=None) -> torch.Tensor:
        """Integrate records [n, nsp+2] = [T, Y_0..Y_{nsp-1}, rho] in place over
        dt (the reference's calcChemODEsArray buffers); subdt is updated in
        place. Returns the per-cell status words."""
        n = TYiRho.shape[0]
        if TYiRho.dim() != 2 or TYiRho.shape[1] != self.nsp + 2:
            raise ValueError("records must be [n, nsp + 2]")
        st = torch.zeros(n, dtype=torch.int32, device=TYiRho.device)
        o = opts if opts is not None else _capi.default_opts()
        rc = _capi.load().hc_integrate_aos(self.handle, C.byref(o), n, _ptr(_f64(TYiRho, "TYiRho")),
                                           _ptr(None if p is None else _f64(p, "p")),
                                           _ptr(_f64(dt, "dt")), _ptr(_f64(subdt, "subdt")),
                                           1 if return_ci else 0, _ptr(st), _stream(stream))
        _capi.check(rc, "hc_integrate_aos")
        return st

    def source_terms_imp(self, T, p, rho, Y, stream=None):
        """(Ri [nsp, n], diag [nsp-1, n]): source terms and the diagonal source
        Jacobian of chemistrySource::calculateSourceTermsImp."""
        n = T.shape[0]
        Ri = torch.empty_like(Y)
        diag = torch.empty((self.nsp - 1, n), dtype=torch.float64, device=T.device)
        rc = _capi.load().hc_source_terms_imp(self.handle, n, _ptr(_f64(T, "T")),
                                              _ptr(_f64(p, "p")), _ptr(_f64(rho, "rho")),
                                              _ptr(_f64(Y, "Y")), _ptr(Ri), _ptr(diag),
                                              _stream(stream))
        _capi.check(rc, "hc_source_terms_imp")
        return Ri, diag

    def temperature_from_enthalpy(self, ha, Y, T0, TLow: float = 50.0, THigh: float = 5000.0,
                                  stream=None):
        """T from the mixture's mass enthalpy (thermoList::THa_p); returns (T, flag)."""
        n = ha.shape[0]
        T = torch.empty_like(_f64(ha, "ha"))
        flag = torch.empty(n, dtype=torch.int32, device=ha.device)
        rc = _capi.load().hc_temperature_from_enthalpy(self.handle, n, _ptr(ha), _ptr(_f64(Y, "Y")),
                                                       _ptr(_f64(T0, "T0")), float(TLow),
                                                       float(THigh), _ptr(T), _ptr(flag),
                                                       _stream(stream))
        _capi.check(rc, "hc_temperature_from_enthalpy")
        return T, flag

    def temperature_from_energy(self, ea, Y, rho, T0, TLow: float = 50.0, THigh: float = 5000.0,
                                stream=None):
        """T from the mixture's mass internal energy at constant density
        (thermoList::TEa_rho); returns (T, flag)."""
        n = ea.shape[0]
        T = torch.empty_like(_f64(ea, "ea"))
        flag = torch.empty(n, dtype=torch.int32, device=ea.device)
        rc = _capi.load().hc_temperature_from_energy(self.handle, n, _ptr(ea), _ptr(_f64(Y, "Y")),
                                                     _ptr(_f64(rho, "rho")), _ptr(_f64(T0, "T0")),
                                                     float(TLow), float(THigh), _ptr(T),
                                                     _ptr(flag), _stream(stream))
        _capi.check(rc, "hc_temperature_from_energy")
        return T, flag

    def properties(self, T, p, Y, stream=None) -> Dict[str, torch.Tensor]:
        """ha [nsp,n] J/kg, cp [n] J/kg/K, mu [n] Pa s, kappa [n] W/m/K, D [nsp,n] m^2/s."""
        n = T.shape[0]
        dev = T.device
        out = {"ha": torch.empty_like(Y), "cp": torch.empty(n, dtype=torch.float64, device=dev),
               "mu": torch.empty(n, dtype=torch.float64, device=dev),
               "kappa": torch.empty(n, dtype=torch.float64, device=dev),
               "D": torch.empty_like(Y)}
        rc = _capi.load().hc_properties(self.handle, n, _ptr(_f64(T, "T")), _ptr(_f64(p, "p")),
                                        _ptr(_f64(Y, "Y")), _ptr(out["ha"]), _ptr(out["cp"]),
                                        _ptr(out["mu"]), _ptr(out["kappa"]), _ptr(out["D"]),
                                        _stream(stream))
        _capi.check(rc, "hc_properties")
        return out


@dataclasses.dataclass
class Flow:
    """Cell fields the chemistry source reads and writes (the reference keeps
    them in flowModel: T(), p(), rho(), mixtures().Yi())."""
    T: torch.Tensor      # [n]
    p: torch.Tensor      # [n]
    rho: torch.Tensor    # [n]
    Y: torch.Tensor      # [nsp, n]

    @property
    def n(self) -> int:
        return int(self.T.shape[0])


class ChemistrySource:
    """B200 drop-in for ODESolver<chemistrySource> with the ImplicitEuler solver."""

    def __init__(self, mech: Mechanism, flow: Flow, **opts):
        self.mech = mech
        self.flow = flow
        self.opts = _capi.default_opts(**opts)
        n = flow.n
        dev = flow.T.device
        self._Ri = torch.zeros((mech.nsp, n), dtype=torch.float64, device=dev)
        self.dtInit: Optional[torch.Tensor] = None   # warm-start sub-steps (chemistrySource.inl:86-95)
        self.status = torch.zeros(n, dtype=torch.int32, device=dev)
        self.cost = torch.zeros(n, dtype=torch.int64, device=dev)
        self.order: Optional[torch.Tensor] = None
        self.rebin = True
        self.last_counters: Dict[str, int] = {}

    def Ri(self, i: Optional[int] = None) -> torch.Tensor:
        return self._Ri if i is None else self._Ri[i]

    def _dt_init(self, dt: torch.Tensor, dt_factor: float) -> torch.Tensor:
        if self.dtInit is None:
            self.dtInit = (dt * dt_factor).clone()
        return self.dtInit

    def _integrate(self, dt: torch.Tensor, dt_factor: float, T, rho, Y, Ri, counters: bool):
        sub = self._dt_init(dt, dt_factor)
        cnt = _capi.HcCounters() if counters else None
        order = self.order if self.rebin else None
        rc = _capi.load().hc_integrate_ordered(
            self.mech.handle, C.byref(self.opts), self.flow.n, _ptr(T), _ptr(self.flow.p),
            _ptr(rho), _ptr(Y), _ptr(_f64(dt, "dt")), float(dt_factor), _ptr(sub), _ptr(Ri),
            _ptr(self.status), _ptr(order), _ptr(self.cost),
            C.addressof(cnt) if cnt is not None else None, _stream())
        _capi.check(rc, "hc_integrate_ordered")
        if cnt is not None:
            self.last_counters = cnt.as_dict()
        if self.rebin:
            # stiffest cells first on the next flow step; updated in place so
            # that a captured graph's launch reads the new order on replay
            new_order = torch.argsort(self.cost, descending=True).to(torch.int32)
            if self.order is None:
                self.order = new_order
            else:
                self.order.copy_(new_order)

    def solve(self, dt: torch.Tensor, dt_factor: float = 1.0, counters: bool = False) -> float:
        """Integrate every cell over dt*dtFactor and fill Ri; the flow fields
        are left unchanged (chemistrySource::solve(dt, dtFactor)). Returns the
        smallest new sub-step."""
        f = self.flow
        T = f.T.clone()
        rho = f.rho.clone()
        Y = f.Y.clone()
        self._integrate(dt, dt_factor, T, rho, Y, self._Ri, counters)
        return float(self.dtInit.min().item())

    def solveUpdate(self, dt: torch.Tensor, dt_factor: float = 1.0, counters: bool = False):
        """Integrate every cell and write Y, T back (chemistrySource::solveUpdate)."""
        f = self.flow
        self._integrate(dt, dt_factor, f.T, f.rho, f.Y, None, counters)

    def capture_update(self, dt: torch.Tensor, dt_factor: float = 1.0) -> "torch.cuda.CUDAGraph":
        """Capture one solveUpdate flow step (queue reset, integrator launch
        and the stiffness re-ordering) in a CUDA graph; replaying it advances
        the flow fields in place. dt, the fields, dtInit and the order buffer
        must stay allocated while the graph is used. A solveUpdate (or solve)
        on these fields must have run first: it sizes the library's per-cell
        buffers (growing them synchronises the stream, which capture forbids)
        and creates the order buffer."""
        if self.dtInit is None or (self.rebin and self.order is None):
            raise RuntimeError("run solveUpdate once before capturing")
        f = self.flow
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                self._integrate(dt, dt_factor, f.T, f.rho, f.Y, None, False)
        torch.cuda.current_stream().wait_stream(side)
        return g

    def calculateSourceTermsImp(self, withoutLastSpec: bool = True):
        """Ri and the diagonal source Jacobian (chemistrySource::calculateSourceTermsImp);
        the diagonal is returned for the first nsp - 1 species, the form the
        flow solver's coupled solve uses (withoutLastSpec = true)."""
        if not withoutLastSpec:
            raise NotImplementedError("only the withoutLastSpec = true form is built")
        f = self.flow
        self._Ri, self.diagSource = self.mech.source_terms_imp(f.T, f.p, f.rho, f.Y)
        return self._Ri, self.diagSource

    def calculateSourceTerms(self, withoutLastSpec: bool = False):
        """Ri = omega_i W_i at the current state (chemistrySource::calculateSourceTerms)."""
        f = self.flow
        self._Ri = self.mech.source_terms(f.T, f.p, f.rho, f.Y)
        return self._Ri


def integrate_host(mech: Mechanism, T: np.ndarray, p: np.ndarray, rho: np.ndarray,
                   Y: np.ndarray, dt: np.ndarray, subdt: Optional[np.ndarray] = None,
                   dt_factor: float = 1.0, Ri: bool = False, **opts):
    """Integrate host (numpy) arrays through hc_integrate_host: copies in,
    integrates, copies out. Arrays are updated in place and returned."""
    n = int(T.shape[0])
    lib = _capi.load()
    o = _capi.default_opts(**opts)
    sub = np.ascontiguousarray(dt if subdt is None else subdt, dtype=np.float64).copy()
    Rout = np.zeros_like(Y) if Ri else None
    status = np.zeros(n, np.int32)
    cnt = _capi.HcCounters()
    vp = lambda a: None if a is None else C.c_void_p(a.ctypes.data)
    rc = lib.hc_integrate_host(mech.handle, C.byref(o), n, vp(T), vp(p), vp(rho), vp(Y), vp(dt),
                               float(dt_factor), vp(sub), vp(Rout), vp(status), C.addressof(cnt),
                               None)
    _capi.check(rc, "hc_integrate_host")
    return {"T": T, "rho": rho, "Y": Y, "subdt": sub, "Ri": Rout, "status": status,
            "counters": cnt.as_dict(), "rc": rc}
