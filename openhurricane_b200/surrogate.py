"""Learned chemistry surrogate: the network (hc_mlp_* of the C ABI) and the
host side of its training and gated inference.

The network maps a cell state and the flow step (T, log p, Y_1..Y_nsp,
log dt), normalised, to the normalised chemistry increment (dT, dY_1..dY_nsp)
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
