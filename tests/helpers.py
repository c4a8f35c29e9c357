"""Helpers shared by the parity tests (device transfers, seeded fields)."""
import numpy as np


def to_dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def to_host(t):
    return t.detach().cpu().numpy()


def rand_spectral(o, seed, scale=1.0):
    """A seeded spectral field of the oracle's shape (no symmetry imposed)."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(o.sshape) + 1j * rng.standard_normal(o.sshape)
    return (scale * a).astype(o.cdt)


def rand_real(o, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(o.rshape).astype(o.rdt)


def solenoidal_ic(o, seed=1000, amp=1.0):
    """Config-0 style initial velocity: random phases, E(k) ~ k^4 exp(-2(k/2)^2)
    on 1 <= |k| <= N/3, <|v|^2> = amp^2."""
    v, _ = o.random_solenoidal(seed, 1.0, o.nx / 3.0, 1, amp)
    return v
