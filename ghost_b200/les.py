"""Host mirror of the LES path: the learned subgrid-stress MLP and the LES
driver with its closures (none, GHOST's EDQNM eddy viscosity, the MLP as a
pointwise stress model or as a spectral eddy viscosity).

`MLP` wraps the ghost_mlp_* entry points (tensor-core forward, gradients and
Adam of the 10 -> 64 -> 64 -> 6 GELU network); inputs and targets are CUDA
float32 tensors of shape (B, 10) and (B, 6).  `LES` wraps ghost_les_*: a
cubic coarse grid (a `Ghost` context) with a sharp cutoff kc.
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


MODELS = {"none": 0, "edqnm": 1, "mlp": 2, "mlp_spectral": 3}


class LES:
    """LES on the coarse grid of `g` (a cubic `Ghost`) resolving |k| <= kc.

    The context's kmax is set to kc^2 so that the LES keeps exactly the
    modes of the sharp-filtered DNS."""

    def __init__(self, g, kc: int):
        self.g = g
        self.lib = g.lib
        self.kc = int(kc)
        check(self.lib.ghost_ctx_set_kmax(g.h, float(self.kc * self.kc)), "ghost_ctx_set_kmax")
        h = ctypes.c_void_p()
        check(self.lib.ghost_les_create(g.h, self.kc, ctypes.byref(h)), "ghost_les_create")
        self.h = h
        self.n = g.nx
        self.model = "none"

    def close(self):
        if getattr(self, "h", None):
            self.lib.ghost_les_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, x):
        return self.g._ptr(x, "c")

    def _f(self, x, cols):
        p = _dev(x, cols, "array")
        if x.shape[0] != self.rows():
            raise ValueError(f"expected {self.rows()} rows (one per grid point), got {x.shape[0]}")
        return p

    def rows(self):
        return self.n ** 3

    def truncate(self, fine, a, out=None):
        """The modes |k| <= kc of a spectrum on `fine` (a Ghost), on this grid."""
        out = self.g.czeros() if out is None else out
        check(self.lib.ghost_les_truncate(self.h, fine.h, fine._ptr(a, "c"), self._c(out)), "ghost_les_truncate")
        return out

    def samples(self, fine, vx, vy, vz, delta: float = 1.0, x=None, tau=None):
        """(inputs (n^3, 10), stresses (n^3, 6)) from a fine velocity."""
        B = self.rows()
        x = torch.empty((B, NIN), dtype=torch.float32, device="cuda") if x is None else x
        tau = torch.empty((B, NOUT), dtype=torch.float32, device="cuda") if tau is None else tau
        check(self.lib.ghost_les_samples(self.h, fine.h, *[fine._ptr(v, "c") for v in (vx, vy, vz)],
                                         ctypes.c_float(delta), self._f(x, NIN), self._f(tau, NOUT)),
              "ghost_les_samples")
        return x, tau

    def features(self, vx, vy, vz, grad_scale: float = 1.0, delta: float = 1.0, x=None):
        x = torch.empty((self.rows(), NIN), dtype=torch.float32, device="cuda") if x is None else x
        check(self.lib.ghost_les_features(self.h, *[self._c(v) for v in (vx, vy, vz)], ctypes.c_float(grad_scale),
                                          ctypes.c_float(delta), self._f(x, NIN)), "ghost_les_features")
        return x

    def spectral_features(self, E, x=None):
        """Inputs of the spectral network, (kc, 10), from a kinetic spectrum
        E: a CUDA float64 tensor of the n/2+1 shell sums (spectrumc, kin = 1)."""
        if not isinstance(E, torch.Tensor) or not E.is_cuda or E.dtype != torch.float64 or E.dim() != 1 \
                or E.shape[0] != self.n // 2 + 1 or not E.is_contiguous():
            raise ValueError(f"E: expected a contiguous CUDA float64 tensor of {self.n // 2 + 1} shells")
        x = torch.empty((self.kc, NIN), dtype=torch.float32, device=E.device) if x is None else x
        p = _dev(x, NIN, "x")
        if x.shape[0] != self.kc:
            raise ValueError(f"x: expected {self.kc} rows, got {x.shape[0]}")
        check(self.lib.ghost_les_spectral_features(self.h, ctypes.c_void_p(E.data_ptr()), p),
              "ghost_les_spectral_features")
        return x

    def tau_force(self, tau, tau_scale: float = 1.0, f=(None, None, None), out=None):
        out = [self.g.czeros() for _ in range(3)] if out is None else out
        check(self.lib.ghost_les_tau_force(self.h, self._f(tau, NOUT), ctypes.c_float(tau_scale),
                                           *[self._c(x) for x in f], *[self._c(x) for x in out]),
              "ghost_les_tau_force")
        return out

    def set_model(self, model: str, mlp: MLP | None = None, grad_scale: float = 1.0, tau_scale: float = 1.0,
                  delta: float = 1.0, kolmo: float = 1.4):
        """Select the closure.  "mlp": the stresses are the network's outputs
        for the inputs (gradients times grad_scale, delta), times tau_scale;
        "mlp_spectral": tve(k) is the network's first output for shell k
        (inputs from spectral_features) times tau_scale sqrt(E(kc)/kc)."""
        check(self.lib.ghost_les_set_model(self.h, MODELS[model], mlp.h if mlp is not None else None,
                                           grad_scale, tau_scale, delta, kolmo), "ghost_les_set_model")
        self.model = model
        self.mlp = mlp

    def set_fallback(self, enable: bool = True, blowup: float = 10.0):
        """Let ``run`` switch the MLP closure to EDQNM when a step diverges."""
        check(self.lib.ghost_les_set_fallback(self.h, int(enable), blowup), "ghost_les_set_fallback")

    def status(self):
        """(selected closure name, step at which the fallback engaged or -1)."""
        m, at = ctypes.c_int(), ctypes.c_longlong()
        check(self.lib.ghost_les_status(self.h, ctypes.byref(m), ctypes.byref(at)), "ghost_les_status")
        return {v: k for k, v in MODELS.items()}[m.value], at.value

    def set_time(self, t: float):
        check(self.lib.ghost_les_set_time(self.h, t), "ghost_les_set_time")

    def closure_force(self, nu, vx, vy, vz, f=(None, None, None), out=None):
        out = [self.g.czeros() for _ in range(3)] if out is None else out
        check(self.lib.ghost_les_closure_force(self.h, nu, *[self._c(v) for v in (vx, vy, vz)],
                                               *[self._c(x) for x in f], *[self._c(x) for x in out]),
              "ghost_les_closure_force")
        return out

    def run(self, nsteps: int, ord: int, dt: float, nu: float, vx, vy, vz, fx=None, fy=None, fz=None):
        check(self.lib.ghost_les_run(self.h, nsteps, ord, dt, nu, *[self._c(v) for v in (vx, vy, vz, fx, fy, fz)]),
              "ghost_les_run")

    def set_helicity(self, heli: int = 1):
        """GHOST's heli flag for the EDQNM closure (full_cusp, tvh, helical vcorrect)."""
        check(self.lib.ghost_les_set_helicity(self.h, int(heli)), "ghost_les_set_helicity")

    def edqnm_last_hel(self):
        """(tvh, thpq, Hk) of the last helical EDQNM evaluation."""
        nb = self.n // 2 + 1
        tvh, thpq, Hk = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        P = ctypes.POINTER(ctypes.c_double)
        check(self.lib.ghost_les_edqnm_last_hel(self.h, tvh.ctypes.data_as(P), thpq.ctypes.data_as(P),
                                                Hk.ctypes.data_as(P)), "ghost_les_edqnm_last_hel")
        return tvh, thpq, Hk

    def edqnm_last(self):
        nb = self.n // 2 + 1
        tve, tepq, Ek = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        P = ctypes.POINTER(ctypes.c_double)
        check(self.lib.ghost_les_edqnm_last(self.h, tve.ctypes.data_as(P), tepq.ctypes.data_as(P),
                                            Ek.ctypes.data_as(P)), "ghost_les_edqnm_last")
        return tve, tepq, Ek


def evedqnm(n: int, kmax: float, Eold, nu: float, time: float, kolmo: float = 1.4, precision: str = "fp64"):
    """GHOST's evedqnm (heli = 0) on the host: (tepq, tve, Ext)."""
    lib = _lib.load()
    nb = n // 2 + 1
    E = np.ascontiguousarray(Eold, dtype=np.float64)
    tepq, tve, Ext = np.zeros(nb), np.zeros(nb), np.zeros(3 * nb)
    P = ctypes.POINTER(ctypes.c_double)
    code = {"fp32": _lib.GHOST_SINGLE, "fp64": _lib.GHOST_DOUBLE}[precision]
    check(lib.ghost_evedqnm(n, code, kmax, kolmo, E.ctypes.data_as(P), nu, time, tepq.ctypes.data_as(P),
                            tve.ctypes.data_as(P), Ext.ctypes.data_as(P)), "ghost_evedqnm")
    return tepq, tve, Ext


def evedqnm_hel(n: int, kmax: float, Eold, Hold, nu: float, time: float, hel: int = 1, kolmo: float = 1.4,
                precision: str = "fp64"):
    """GHOST's evedqnm with its hel flag on the host:
    (tepq, thpq, tve, tvh, Ext, Hxt)."""
    lib = _lib.load()
    nb = n // 2 + 1
    E = np.ascontiguousarray(Eold, dtype=np.float64)
    H = np.ascontiguousarray(Hold, dtype=np.float64)
    out = [np.zeros(nb) for _ in range(4)] + [np.zeros(3 * nb), np.zeros(3 * nb)]
    P = ctypes.POINTER(ctypes.c_double)
    code = {"fp32": _lib.GHOST_SINGLE, "fp64": _lib.GHOST_DOUBLE}[precision]
    check(lib.ghost_evedqnm_hel(n, code, kmax, kolmo, E.ctypes.data_as(P), H.ctypes.data_as(P), nu, time, int(hel),
                                *[x.ctypes.data_as(P) for x in out]), "ghost_evedqnm_hel")
    return tuple(out)


__all__ = ["MLP", "LES", "evedqnm", "evedqnm_hel", "MODELS", "NIN", "NHID", "NOUT", "NPARAM"]
