"""Host mirror of the LES closures: the learned subgrid-stress MLP.

`MLP` wraps the ghost_mlp_* entry points (tensor-core forward, gradients and
Adam of the 10 -> 64 -> 64 -> 6 GELU network).  Inputs and targets are CUDA
float32 tensors of shape (B, 10) and (B, 6).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check

try:
    import torch
except Exception:  # pragma: no cover
    torch = None

NIN, NHID, NOUT, NPARAM = 10, 64, 6, 5254


def _dev(x, cols, name):
    if torch is None or not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ValueError(f"{name}: expected a CUDA tensor")
    if x.dtype != torch.float32 or x.dim() != 2 or x.shape[1] != cols or not x.is_contiguous():
        raise ValueError(f"{name}: expected contiguous float32 (B, {cols}), got {x.dtype} {tuple(x.shape)}")
    return ctypes.c_void_p(x.data_ptr())


class MLP:
    """The subgrid-stress network on the current CUDA device."""

    def __init__(self, seed: int = 0, stream=None):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        check(self.lib.ghost_mlp_create(int(seed), ctypes.byref(h)), "ghost_mlp_create")
        self.h = h
        if stream is None and torch is not None and torch.cuda.is_available():
            stream = torch.cuda.current_stream().cuda_stream
        if stream is not None:
            check(self.lib.ghost_mlp_set_stream(self.h, ctypes.c_void_p(stream)), "ghost_mlp_set_stream")

    def close(self):
        if getattr(self, "h", None):
            self.lib.ghost_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.empty(NPARAM, np.float32)
        check(self.lib.ghost_mlp_get_params(self.h, p.ctypes.data_as(ctypes.c_void_p)), "ghost_mlp_get_params")
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (NPARAM,):
            raise ValueError(f"expected {NPARAM} parameters")
        check(self.lib.ghost_mlp_set_params(self.h, p.ctypes.data_as(ctypes.c_void_p)), "ghost_mlp_set_params")

    def forward(self, x, y=None):
        if y is None:
            y = torch.empty((x.shape[0], NOUT), dtype=torch.float32, device=x.device)
        check(self.lib.ghost_mlp_forward(self.h, _dev(x, NIN, "x"), _dev(y, NOUT, "y"), int(x.shape[0])),
              "ghost_mlp_forward")
        return y

    def gradients(self, x, t):
        """(gradient vector float32[NPARAM], loss) without an update."""
        g = np.empty(NPARAM, np.float32)
        loss = ctypes.c_double()
        check(self.lib.ghost_mlp_gradients(self.h, _dev(x, NIN, "x"), _dev(t, NOUT, "t"), int(x.shape[0]),
                                           g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(loss)),
              "ghost_mlp_gradients")
        return g, loss.value

    def train_step(self, x, t, lr: float, want_loss: bool = True):
        loss = ctypes.c_double()
        check(self.lib.ghost_mlp_train_step(self.h, _dev(x, NIN, "x"), _dev(t, NOUT, "t"), int(x.shape[0]),
                                            ctypes.c_float(lr), ctypes.byref(loss) if want_loss else None),
              "ghost_mlp_train_step")
        return loss.value if want_loss else None


__all__ = ["MLP", "NIN", "NHID", "NOUT", "NPARAM"]
