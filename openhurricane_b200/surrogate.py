"""Learned chemistry surrogate: the network (hc_mlp_* of the C ABI) and the
host side of its training and gated inference.

The network maps a cell state and the flow step (T, ln p, ln Y_1..ln Y_nsp,
ln dt), normalised, to the normalised chemistry increment (dT, dY_1..dY_nsp)
over that step. Its forward and backward passes are the library's BF16
tcgen05 kernels accumulating in FP32; parameters are FP32 with Adam.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _capi


def _vp(t: Optional[torch.Tensor]):
    return None if t is None else C.c_void_p(t.data_ptr())


def _f32(t: torch.Tensor, name: str) -> torch.Tensor:
    if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
    return t


class MLP:
    """n_in -> n_hidden x width (GELU) -> n_out on the GPU."""

    def __init__(self, n_in: int, n_out: int, n_hidden: int, width: int, max_batch: int = 8192,
                 seed: int = 0):
        self.n_in, self.n_out, self.n_hidden, self.width = n_in, n_out, n_hidden, width
        self.max_batch = max_batch
        lib = _capi.load()
        h = C.c_void_p()
        _capi.check(lib.hc_mlp_create(n_in, n_out, n_hidden, width, max_batch, seed, C.byref(h)),
                    "hc_mlp_create")
        self.handle = h
        self.n_params = int(lib.hc_mlp_num_params(h))

    def close(self):
        if getattr(self, "handle", None):
            _capi.load().hc_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shapes(self):
        dims = [self.n_in] + [self.width] * self.n_hidden + [self.n_out]
        return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        _capi.check(_capi.load().hc_mlp_get_params(self.handle, C.c_void_p(out.ctypes.data)),
                    "hc_mlp_get_params")
        return out

    def set_params(self, theta: np.ndarray):
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        if theta.size != self.n_params:
            raise ValueError("parameter vector has the wrong size")
        _capi.check(_capi.load().hc_mlp_set_params(self.handle, C.c_void_p(theta.ctypes.data)),
                    "hc_mlp_set_params")

    def grad(self, X: torch.Tensor, Y: torch.Tensor):
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float(0.0)
        _capi.check(_capi.load().hc_mlp_grad(self.handle, _vp(_f32(X, "X")), _vp(_f32(Y, "Y")),
                                             int(X.shape[0]), C.c_void_p(g.ctypes.data),
                                             C.byref(loss), _vp_stream()), "hc_mlp_grad")
        return float(loss.value), g

    def train_step(self, X: torch.Tensor, Y: torch.Tensor, lr: float, want_loss: bool = False,
                   check: bool = False) -> Optional[float]:
        loss = C.c_float(0.0)
        _capi.check(_capi.load().hc_mlp_train_step(
            self.handle, _vp(_f32(X, "X")), _vp(_f32(Y, "Y")), int(X.shape[0]), float(lr),
            C.byref(loss) if want_loss else None, 1 if check else 0, _vp_stream()),
            "hc_mlp_train_step")
        return float(loss.value) if want_loss else None

    def forward(self, X: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        X = _f32(X, "X")
        if out is None:
            out = torch.empty((X.shape[0], self.n_out), dtype=torch.float32, device=X.device)
        _capi.check(_capi.load().hc_mlp_forward(self.handle, _vp(X), int(X.shape[0]), _vp(out),
                                                _vp_stream()), "hc_mlp_forward")
        return out

    def check(self):
        _capi.check(_capi.load().hc_mlp_check(self.handle, _vp_stream()), "hc_mlp_check")


def _vp_stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def gemm_bf16(A: torch.Tensor, B: torch.Tensor, bias: Optional[torch.Tensor] = None,
              act: int = 0) -> torch.Tensor:
    """C = act(A B^T + bias) on the tensor cores (test entry)."""
    if A.dtype != torch.bfloat16 or B.dtype != torch.bfloat16:
        raise ValueError("A and B must be bfloat16")
    M, K = A.shape
    N = B.shape[0]
    Cm = torch.empty((M, N), dtype=torch.float32, device=A.device)
    _capi.check(_capi.load().hc_gemm_bf16_tn(_vp(A.contiguous()), _vp(B.contiguous()), M, N, K,
                                             _vp(bias), act, _vp(Cm), _vp_stream()),
                "hc_gemm_bf16_tn")
    return Cm


def element_projector(tables) -> np.ndarray:
    """P = I - A^T (A A^T)^+ A with A[e][i] = atoms of element e in species i
    / W_i: P dY conserves every element's mass (and so sum dY = 0)."""
    A = tables.elem_matrix / tables.W[None, :]
    A = A[np.abs(A).sum(axis=1) > 0]
    nsp = tables.nsp
    P = np.eye(nsp) - A.T @ np.linalg.pinv(A @ A.T) @ A
    return np.ascontiguousarray(P)


class Surrogate:
    """Gated learned chemistry step for one mechanism.

    The network predicts the normalised increment (dT, dY) of a flow step
    from the normalised (T, ln p, Y, ln dt); the FP64 gate
    (hc_surrogate_gate) projects dY onto element conservation, recovers T
    from the conserved enthalpy and accepts or rejects each cell; rejected
    cells are integrated by the FP64 integrator (hc_integrate_subset)."""

    def __init__(self, mech, n_hidden: int = 3, width: int = 256, max_batch: int = 65536,
                 seed: int = 0, n_ensemble: int = 3):
        self.mech = mech
        t = mech.tables
        self.nsp = t.nsp
        self.n_in, self.n_out = t.nsp + 3, t.nsp + 1
        # an ensemble of networks trained from different initialisations and
        # batch orders: their disagreement is the gate's confidence measure
        self.nets = [MLP(self.n_in, self.n_out, n_hidden, width, max_batch=max_batch,
                         seed=seed + 1000 * k) for k in range(n_ensemble)]
        self.net = self.nets[0]
        # disagreement scales: a cell is rejected when the ensemble's spread
        # in dT exceeds spread_T (K) or in any dY exceeds spread_Y
        self.spread_T = 1.0
        self.spread_Y = 1e-2
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        self.proj = torch.tensor(element_projector(t), dtype=torch.float64, device=dev)
        A = t.elem_matrix / t.W[None, :]
        A = A[np.abs(A).sum(axis=1) > 0]
        self.elem = torch.tensor(np.ascontiguousarray(A), dtype=torch.float64, device=dev)
        self.nel = int(A.shape[0])
        self.in_mean = torch.zeros(self.n_in, dtype=torch.float64, device=dev)
        self.in_istd = torch.ones(self.n_in, dtype=torch.float64, device=dev)
        self.out_mean = torch.zeros(self.n_out, dtype=torch.float64, device=dev)
        self.out_std = torch.ones(self.n_out, dtype=torch.float64, device=dev)
        self.gate = _capi.HcGateOpts(tol_T=2.0, tol_proj=0.5, y_neg=1e-4, x_max=8.0, T_min=250.0,
                                     T_max=4000.0, tol_spread=1.0)

    # ------------------------------------------------------------------ data
    def features(self, T, p, Y, dt, dt_factor: float = 1.0, out=None) -> torch.Tensor:
        n = int(T.shape[0])
        X = out if out is not None else torch.empty((n, self.n_in), dtype=torch.float32,
                                                    device=T.device)
        _capi.check(_capi.load().hc_surrogate_features(
            self.mech.handle, n, _vp(T), _vp(p), _vp(Y), _vp(dt), float(dt_factor),
            _vp(self.in_mean), _vp(self.in_istd), _vp(X), _vp_stream()),
            "hc_surrogate_features")
        return X

    @staticmethod
    def raw_features(T, p, Y, dt):
        """(T, ln p, ln max(Y_i, 1e-20), ln dt) per cell, as hc_surrogate_features."""
        lY = torch.log(torch.clamp(Y, min=1e-20))
        return torch.cat([T[None], torch.log(p)[None], lY, torch.log(dt)[None]], dim=0).T

    def fit_normalisation(self, T, p, Y, dt, dT, dY):
        """Input / output statistics of the training set (float64)."""
        raw = self.raw_features(T, p, Y, dt)
        mu, sd = raw.mean(0), raw.std(0)
        self.in_mean = mu.contiguous()
        self.in_istd = torch.where(sd > 1e-12, 1.0 / sd, torch.ones_like(sd)).contiguous()
        d = torch.cat([dT[None], dY], dim=0).T
        self.out_mean = d.mean(0).contiguous()
        osd = d.std(0)
        self.out_std = torch.where(osd > 1e-30, osd, torch.ones_like(osd)).contiguous()

    def targets(self, dT, dY) -> torch.Tensor:
        d = torch.cat([dT[None], dY], dim=0).T
        return ((d - self.out_mean) / self.out_std).to(torch.float32).contiguous()

    # ------------------------------------------------------------------ train
    def train(self, X: torch.Tensor, D: torch.Tensor, epochs: int = 150, batch: int = 8192,
              lr: float = 2e-3, lr_final: float = 2e-5, seed: int = 0, log=None):
        """Adam over shuffled mini-batches with a cosine learning-rate decay,
        every network of the ensemble with its own batch order. Returns the
        first network's loss at the end of each epoch."""
        n = int(X.shape[0])
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        losses = []
        for m, net in enumerate(self.nets):
            g = torch.Generator(device=X.device).manual_seed(seed + 7919 * m)
            k = 0
            for ep in range(epochs):
                perm = torch.randperm(n, device=X.device, generator=g)
                for s in range(steps_per_epoch):
                    idx = perm[s * batch:(s + 1) * batch]
                    xb, yb = X[idx].contiguous(), D[idx].contiguous()
                    a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(1, total)))
                    want = (s == steps_per_epoch - 1) and (m == 0 or ep == epochs - 1)
                    l = net.train_step(xb, yb, a, want_loss=want, check=want)
                    if want and m == 0:
                        losses.append(l)
                        if log:
                            log(f"epoch {ep} loss {l:.4e}")
                    k += 1
        return losses

    def predict(self, X: torch.Tensor):
        """Mean normalised prediction of the ensemble and its per-cell
        disagreement (the larger of the dT spread / spread_T and the largest
        dY spread / spread_Y; <= 1 is confident)."""
        preds = torch.stack([net.forward(X) for net in self.nets])
        mean = preds.mean(dim=0).contiguous()
        if len(self.nets) == 1:
            return mean, None
        rng = (preds.max(dim=0).values - preds.min(dim=0).values).double() * self.out_std[None, :]
        sp = torch.maximum(rng[:, 0] / self.spread_T, rng[:, 1:].max(dim=1).values / self.spread_Y)
        return mean, sp.to(torch.float32).contiguous()

    # ------------------------------------------------------------------ infer
    def step(self, flow, dt: torch.Tensor, dt_factor: float = 1.0, opts=None,
             subdt: Optional[torch.Tensor] = None, counters: Optional[dict] = None):
        """One gated surrogate flow step on `flow` (T, p, rho, Y updated in
        place). Returns (n_rejected, accept mask). `counters`, when given, is
        filled with the FP64 fallback's work counters (n_newton, ...; zeros
        when no cell is rejected)."""
        n = flow.n
        X = self.features(flow.T, flow.p, flow.Y, dt, dt_factor)
        pred, spread = self.predict(X)
        return self.apply(flow, dt, X, pred, spread, dt_factor, opts, subdt, counters)

    def apply(self, flow, dt, X, pred, spread, dt_factor: float = 1.0, opts=None, subdt=None,
              counters: Optional[dict] = None):
        """The gate and the FP64 fallback for a given prediction."""
        n = flow.n
        accept = torch.empty(n, dtype=torch.int32, device=flow.T.device)
        rejected = torch.empty(n, dtype=torch.int32, device=flow.T.device)
        nrej = C.c_int64(0)
        _capi.check(_capi.load().hc_surrogate_gate(
            self.mech.handle, n, _vp(flow.T), _vp(flow.p), _vp(flow.rho), _vp(flow.Y), _vp(pred),
            _vp(X), _vp(self.out_mean), _vp(self.out_std), _vp(self.proj), _vp(self.elem),
            self.nel, _vp(spread), C.byref(self.gate), _vp(accept), _vp(rejected), C.byref(nrej),
            _vp_stream()),
            "hc_surrogate_gate")
        nr = int(nrej.value)
        cnt = _capi.HcCounters() if counters is not None else None
        if nr > 0:
            o = opts if opts is not None else _capi.default_opts()
            sub = subdt if subdt is not None else (dt * dt_factor).clone()
            _capi.check(_capi.load().hc_integrate_subset(
                self.mech.handle, C.byref(o), n, nr, _vp(rejected), _vp(flow.T), _vp(flow.p),
                _vp(flow.rho), _vp(flow.Y), _vp(dt), float(dt_factor), _vp(sub), None, None, None,
                C.addressof(cnt) if cnt is not None else None, _vp_stream()), "hc_integrate_subset")
        if counters is not None:
            counters.update(cnt.as_dict())
        return nr, accept


def integrate_device(mech, T, p, rho, Y, dt, opts=None):
    """FP64 integration of device arrays over per-cell dt (in place);
    returns the per-cell status."""
    n = int(T.shape[0])
    o = opts if opts is not None else _capi.default_opts()
    sub = dt.clone()
    status = torch.zeros(n, dtype=torch.int32, device=T.device)
    _capi.check(_capi.load().hc_integrate(mech.handle, C.byref(o), n, _vp(T), _vp(p), _vp(rho),
                                          _vp(Y), _vp(dt), 1.0, _vp(sub), None, _vp(status), None,
                                          _vp_stream()), "hc_integrate")
    return status


def generate_samples(mech, T, p, rho, Y, dt_nominal: float, n_samples: int, seed: int = 0,
                     t_max: Optional[float] = None, dt_spread: float = 3.0, opts=None):
    """Training samples for the surrogate from the FP64 GPU integrator.

    Starting states (T, p, rho, Y: device arrays of base cells) are tiled to
    n_samples; half of them are advanced along their own reaction
    trajectories by a random time in [0, t_max] (default: one flow step, so
    that states part-way through a step of ignition appear), and every
    sample is then integrated over a flow step dt drawn log-uniformly in
    [dt_nominal / dt_spread, dt_nominal * dt_spread]. Returns the pre-step
    state, dt and the increments (dT, dY)."""
    if t_max is None:
        t_max = dt_nominal
    dev = T.device
    g = torch.Generator(device=dev).manual_seed(seed)
    nb = int(T.shape[0])
    idx = torch.randint(0, nb, (n_samples,), device=dev, generator=g)
    T1, p1, r1 = T[idx].contiguous(), p[idx].contiguous(), rho[idx].contiguous()
    Y1 = Y[:, idx].contiguous()
    tau = torch.rand(n_samples, device=dev, dtype=torch.float64, generator=g) * t_max
    tau = torch.where(tau < 1e-9, torch.full_like(tau, 1e-9), tau)
    # half of the samples stay at their drawn state (tau tiny), half move along
    keep = torch.rand(n_samples, device=dev, generator=g) < 0.5
    tau = torch.where(keep, torch.full_like(tau, 1e-12), tau)
    integrate_device(mech, T1, p1, r1, Y1, tau, opts)
    u = torch.rand(n_samples, device=dev, dtype=torch.float64, generator=g)
    dt = dt_nominal * torch.exp((2.0 * u - 1.0) * np.log(dt_spread))
    T2, r2, Y2 = T1.clone(), r1.clone(), Y1.clone()
    st = integrate_device(mech, T2, p1, r2, Y2, dt, opts)
    good = (st & 12) == 0
    sel = torch.nonzero(good).flatten()
    return {"T": T1[sel].contiguous(), "p": p1[sel].contiguous(), "rho": r1[sel].contiguous(),
            "Y": Y1[:, sel].contiguous(), "dt": dt[sel].contiguous(),
            "dT": (T2 - T1)[sel].contiguous(), "dY": (Y2 - Y1)[:, sel].contiguous()}
