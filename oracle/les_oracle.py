"""CPU restatement of the LES data path and closure forces.

TEST INFRASTRUCTURE ONLY: tests/ use it as the checker of ghost_b200's LES
kernels (ghost_b200/csrc/les.cu).  The product never imports it.

Built on the oracle's GHOST restatement (oracle.py): its unnormalised
transforms, derivk3 and the sharp-cutoff truncation o_les_truncate (GHOST's
sharp of pseudo/pseudospec3D_filt.f90:200-241 with Delta = pi/kc, then the
N^3 -> n^3 truncation of analysis/trunc3D.fpp).  The subgrid stress is the
standard one, tau_ab = filt(u_a u_b) - ubar_a ubar_b, evaluated at the
coarse grid points; the closure force is -P div tau.

Sample rows follow the real layout r(i,j,k), x fastest, i.e. numpy's
C-order flattening of shape (nz, ny, nx).
"""
from __future__ import annotations

import numpy as np

PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]


def features(co, v, grad_scale=1.0, delta=1.0):
    """Closure inputs of a coarse velocity: x[q][3a+b] = du_a/dx_b * grad_scale, x[q][9] = delta."""
    n3 = co.nx * co.ny * co.nz
    x = np.zeros((n3, 10))
    for a in range(3):
        for b in range(3):
            g = co.fftp3d_complex_to_real(co.derivk3(v[a], b + 1)) / n3
            x[:, 3 * a + b] = g.ravel() * grad_scale
    x[:, 9] = delta
    return x


def samples(fo, co, v, kc, delta=1.0):
    """(inputs, stresses) at the coarse grid points from a fine velocity."""
    N3 = fo.nx * fo.ny * fo.nz
    n3 = co.nx * co.ny * co.nz
    ub = [fo.les_truncate(co, x, kc) for x in v]
    x = features(co, ub, 1.0, delta)
    ur = [co.fftp3d_complex_to_real(u) / n3 for u in ub]
    U = [fo.fftp3d_complex_to_real(u) / N3 for u in v]
    tau = np.zeros((n3, 6))
    for m, (a, b) in enumerate(PAIRS):
        ph = fo.les_truncate(co, fo.fftp3d_real_to_complex(U[a] * U[b]), kc)
        p = co.fftp3d_complex_to_real(ph) / n3
        tau[:, m] = (p - ur[a] * ur[b]).ravel()
    return x, tau


def tau_force(co, tau, tau_scale=1.0, f=None):
    """o = f + P(-i k_b T_ab) on tiny <= kn2 <= kmax (f elsewhere)."""
    kx, ky, kz, kn2, _ = co.tables()
    nxh = co.nxh
    K = [kx[:nxh][:, None, None], ky[None, :, None], kz[None, None, :]]
    T = {}
    for m, (a, b) in enumerate(PAIRS):
        r = (tau[:, m] * tau_scale).reshape(co.rshape)
        T[(a, b)] = T[(b, a)] = co.fftp3d_real_to_complex(r)
    F = [sum(-1j * K[b] * T[(a, b)] for b in range(3)) for a in range(3)]
    kk2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    mask = (kn2 <= co.kmax) & (kn2 >= co.tiny)
    with np.errstate(invalid="ignore", divide="ignore"):
        d = (K[0] * F[0] + K[1] * F[1] + K[2] * F[2]) / kk2
    out = []
    for a in range(3):
        Fa = np.where(mask, F[a] - K[a] * d, 0)
        out.append(Fa + (f[a] if f is not None else 0))
    return out


def eddy_force(co, v, tve, f=None, tvh=None):
    """o = f - tve(ki) kk2 v (+ tvh(ki) curl v, the helical closure of
    include/edqnmhd_rkstep2.f90:45-56) with ki = int(sqrt(kk2) + 0.501) on
    tiny <= kn2 <= kmax."""
    _, _, _, kn2, kk2 = co.tables()
    mask = (kn2 <= co.kmax) & (kn2 >= co.tiny)
    ki = (np.sqrt(kk2) + np.float32(0.501)).astype(int)
    pick = lambda t: np.where(mask & (ki >= 1) & (ki <= len(t)), np.asarray(t)[np.clip(ki - 1, 0, len(t) - 1)], 0.0)
    nut = pick(tve)
    out = [-(nut * np.where(mask, kk2, 0)) * x + (f[a] if f is not None else 0) for a, x in enumerate(v)]
    if tvh is not None:
        nuh = pick(tvh)
        w = [co.rotor3(v[1], v[2], 1), co.rotor3(v[0], v[2], 2), co.rotor3(v[0], v[1], 3)]
        out = [o + nuh * x for o, x in zip(out, w)]
    return out


def helical(co, v, sign=1):
    """The helical part of a solenoidal spectral field: (v + sign i k x v / |k|) / 2,
    a field of helicity density of one sign (zero at k = 0)."""
    kx, ky, kz, _, kk2 = co.tables()
    kx = kx[:co.nxh][:, None, None]
    ky = ky[None, :, None]
    kz = kz[None, None, :]
    kn = np.sqrt(np.where(kk2 > 0, kk2, 1.0))
    cx = 1j * (ky * v[2] - kz * v[1])
    cy = 1j * (kz * v[0] - kx * v[2])
    cz = 1j * (kx * v[1] - ky * v[0])
    h = [0.5 * (a + sign * b / kn) for a, b in zip(v, (cx, cy, cz))]
    return [np.where(kk2 > 0, x, 0).astype(co.cdt) for x in h]


def spectral_features(E, kc):
    """Inputs of the spectral network (kc rows of 10, float32) from the shell
    sums E (E[k-1] the shell k), as ghost_les_spectral_features defines them."""
    E = np.asarray(E, dtype=np.float64)
    tot = float(np.sum(np.maximum(E[:kc], 0.0)))
    fl = 1e-30 * max(tot, 1e-300)
    e = lambda k: max(E[k - 1], fl)  # noqa: E731
    ec = e(kc)
    kh = max(kc // 2, 1)
    slope_c = np.log(ec / e(kh)) / np.log(kc / kh) if kh < kc else 0.0
    frac = np.log(kc * ec / max(tot, fl))
    x = np.zeros((kc, 10))
    for k in range(1, kc + 1):
        r = k / kc
        ka, kb = (k - 1 if k > 1 else k), (k + 1 if k < kc else k)
        sl = np.log(e(kb) / e(ka)) / np.log(kb / ka) if ka < kb else 0.0
        x[k - 1, :8] = [r, r * r, np.log(e(k) / ec) / 8.0, sl / 4.0, slope_c / 4.0, frac / 8.0,
                        np.exp(-(kc - k) / 2.0), np.exp(-(kc - k) / 8.0)]
    return x.astype(np.float32)


def spectral_tve(y0, E, kc, nb, out_scale):
    """tve of the spectral closure: max(y0[k-1] out_scale sqrt(E(kc)/kc), 0)
    for k <= kc, 0 beyond."""
    s = out_scale * np.sqrt(max(float(E[kc - 1]), 0.0) / kc)
    t = np.zeros(nb)
    t[:kc] = np.maximum(np.asarray(y0, dtype=np.float64)[:kc] * s, 0.0)
    return t
