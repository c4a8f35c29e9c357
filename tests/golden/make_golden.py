"""Generates the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

GHOST ships no golden vectors or known-answer files for its HD path, so the
fixtures are produced by the oracle (a restatement of GHOST's FFTW/OpenMP
double-precision path) on seeded inputs and committed, so that the GPU tests
can check the CUDA library without the oracle's build and the CPU tests can
check that the oracle has not drifted.

Files (numpy .npz, all FP64 unless noted):
  hd64_cfg0.npz    64^3 decaying HD, seed 1000, E(k) ~ k^4 exp(-2(k/2)^2) on
                   1 <= |k| <= 64/3 with <|v|^2> = 1, nu = 2e-3, dt = 1e-3,
                   RK2, no forcing.  After 0, 1, 10 and 100 steps: energy
                   (kin 1), enstrophy (kin 0), helicity, the kinetic shell
                   spectrum, the L2 norm of every kx plane of each component,
                   and the modes with kx < 8 and |ky|, |kz| < 8 (3, 8, 16, 16).
  hd16_forced.npz  16^3 forced HD, the 512^3 forced recipe at small size
                   (forcing on 2 <= |k| <= 3 with <|f|^2> = 1, nu = 1e-3,
                   dt = 5e-4, RK4): full fields after 0 and 5 steps.
  bouss16.npz      16^3 rotating stratified Boussinesq on the
                   elongated box (1, 1, 1/4), omegaz 0.5, N = 8, nu = kappa =
                   5e-4, RK4, dt = 2.5e-4: full fields after 3 steps.
  fft.npz          r2c of seeded real fields (16^3 and 32 x 16 x 16) and c2r
                   of the results.
  mlp.npz          the subgrid-stress MLP: parameters, 256 inputs and
                   targets, outputs, loss and gradients (exact FP64 and with
                   the kernels' BF16 operand rounding), FP32 where stored so.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def low_modes(a, m=8):
    """Modes kx < m, ky and kz in [-m, m) of a spectral field (nxh, ny, nz)."""
    idx = np.r_[0:m, -m:0]
    return a[:m][:, idx][:, :, idx]


def plane_norms(a):
    return np.sqrt(np.sum(np.abs(a) ** 2, axis=(1, 2)))


def hd64_cfg0(Oracle):
    o = Oracle(64)
    v, _ = o.random_solenoidal(1000, 1.0, 64 / 3.0, 1, 1.0)
    out = {}
    done = 0
    for n in (0, 1, 10, 100):
        if n > done:
            v = o.hd_run(n - done, 2, 1e-3, 2e-3, v)
            done = n
        Ek, Hk = o.spectrumc(*v, 1, 1)
        out[f"E_{n}"] = o.energy(*v, 1)
        out[f"W_{n}"] = o.energy(*v, 0)
        out[f"H_{n}"] = o.helicity(*v)
        out[f"Ek_{n}"] = Ek
        out[f"planes_{n}"] = np.stack([plane_norms(x) for x in v])
        out[f"modes_{n}"] = np.stack([low_modes(x) for x in v])
    return out


def hd16_forced(Oracle):
    o = Oracle(16)
    v, _ = o.random_solenoidal(1000, 1.0, 16 / 3.0, 1, 1.0)
    f, _ = o.random_solenoidal(2000, 2.0, 3.0, 0, 1.0)
    v5 = o.hd_run(5, 4, 5e-4, 1e-3, v, f)
    return {"v0": np.stack(v), "f": np.stack(f), "v5": np.stack(v5)}


def bouss16(Oracle):
    o = Oracle(16, 16, 16, 1.0, 1.0, 0.25, arbsize=True)
    v, _ = o.random_solenoidal(1000, 2.0, 4.0, 0, 1.0)
    th = o.czeros()
    v3, th3 = o.bouss_run(3, 4, 2.5e-4, 5e-4, 5e-4, 0.5, 8.0, 8.0, v, th)
    return {"v0": np.stack(v), "v3": np.stack(v3), "th3": th3}


def fft(Oracle):
    out = {}
    for tag, shape in (("a", (16, 16, 16)), ("b", (32, 16, 16))):
        o = Oracle(*shape)
        r = np.random.default_rng(77).standard_normal(o.rshape)
        c = o.fftp3d_real_to_complex(r)
        out[f"r_{tag}"] = r
        out[f"c_{tag}"] = c
        out[f"rr_{tag}"] = o.fftp3d_complex_to_real(c.copy())
    return out


def mlp():
    from oracle import mlp_oracle as M
    p = M.glorot(2026)
    rng = np.random.default_rng(2027)
    x = rng.standard_normal((256, M.NIN)).astype(np.float32)
    t = (0.5 * rng.standard_normal((256, M.NOUT))).astype(np.float32)
    ge, le = M.gradients(p, x, t, emulate=True)
    gx, lx = M.gradients(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    return {"params": p, "x": x, "t": t, "y_bf16": M.forward(p, x, emulate=True),
            "y_exact": M.forward(p.astype(np.float64), x.astype(np.float64)),
            "grad_bf16": ge, "loss_bf16": le, "grad_exact": gx, "loss_exact": lx}


def generate():
    from oracle.oracle import Oracle, build
    build()
    return {"hd64_cfg0": hd64_cfg0(Oracle), "hd16_forced": hd16_forced(Oracle), "bouss16": bouss16(Oracle),
            "fft": fft(Oracle), "mlp": mlp()}


def main():
    for name, d in generate().items():
        np.savez(os.path.join(HERE, name + ".npz"), **d)
        print(name, sum(np.asarray(x).nbytes for x in d.values()), "bytes")


if __name__ == "__main__":
    main()
