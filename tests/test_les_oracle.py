"""LES pieces on the CPU: the library's host EDQNM (ghost_evedqnm, no GPU
needed) against the oracle's restatement of pseudo/pseudospec3D_edqnm.f90,
the oracle's EDQNM against the properties of the closure, and the sample
and force restatements against identities of the filtered equations."""
import numpy as np
import pytest

from oracle import les_oracle as LO
from oracle.oracle import Oracle
from tests.conftest import rel_l2


def kolmogorov(n, kc, s=0.02):
    k = np.arange(1, n // 2 + 2, dtype=float)
    E = k ** (-5 / 3) * np.exp(-s * k)
    E[kc:] = 0
    return E


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n,kc", [(64, 21), (128, 42)])
def test_library_evedqnm_matches_oracle(prec, n, kc):
    from ghost_b200.les import evedqnm
    o = Oracle(n, precision=prec)
    o.set_kmax(float(kc * kc))
    E = kolmogorov(n, kc)
    for t in (0.05, 0.5, 5.0):
        ref = o.evedqnm(E, 1e-3, t)
        got = evedqnm(n, float(kc * kc), E, 1e-3, t, precision=prec)
        tol = 1e-12 if prec == "fp64" else 1e-5
        for a, b in zip(got, ref):
            assert rel_l2(a, b) <= tol


def test_edqnm_eddy_viscosity_shape():
    """Positive, cusp-shaped eddy viscosity (rising towards kc); no closure
    at t = 0 (theta cancels frac) and none when the fit fails."""
    o = Oracle(128)
    o.set_kmax(42.0 ** 2)
    E = kolmogorov(128, 42)
    _, tve, Ext = o.evedqnm(E, 1e-4, 10.0)
    assert np.all(tve[:42] > 0) and np.all(tve[42:] == 0)
    assert tve[41] > 3 * tve[20]
    assert np.all(Ext[42:126] > 0) and np.all(np.diff(Ext[42:126]) < 0)
    _, tve0, _ = o.evedqnm(E, 1e-4, 0.0)
    assert np.all(tve0 == 0)
    steep = np.exp(-np.arange(1, 66, dtype=float))  # power < 0: no fit, no closure
    _, tve1, _ = o.evedqnm(steep, 1e-4, 10.0)
    assert np.all(tve1 == 0)


def test_samples_identities():
    """tau from a field that is already band-limited to kc is zero, and the
    features are the exact gradients of the filtered field."""
    fo, co = Oracle(32), Oracle(16)
    kc = 3
    v, _ = fo.random_solenoidal(5, 1.0, 3.0, 0, 1.0)
    # a field with |k| <= 1.5 squares to |k| <= 3 = kc: the filter keeps all of u_a u_b
    vlow, _ = fo.random_solenoidal(6, 1.0, 1.5, 0, 1.0)
    x, tau = LO.samples(fo, co, vlow, kc)
    assert np.max(np.abs(tau)) < 1e-13 * np.max(np.abs(x[:, :9])) ** 2
    # with kc = 2 part of v (|k| <= 3) is unresolved: the mean trace of tau is
    # the energy of the removed modes, <|u|^2> - <|ubar|^2>
    x, tau = LO.samples(fo, co, v, 2)
    assert np.max(np.abs(tau)) > 1e-3
    kx, ky, kz, kn2, kk2 = fo.tables()
    w = np.where(np.arange(fo.nxh)[:, None, None] == 0, 1.0, 2.0)
    removed = sum(np.sum(w * np.abs(np.where(kk2 > 4, a, 0)) ** 2) for a in v) / (32 ** 3) ** 2
    assert abs(np.mean(tau[:, 0] + tau[:, 1] + tau[:, 2]) - removed) < 1e-12 * removed
    # solenoidal filtered field: the trace of the gradient vanishes pointwise
    assert np.max(np.abs(x[:, 0] + x[:, 4] + x[:, 8])) < 1e-12


def test_tau_force_is_solenoidal_and_matches_divergence():
    co = Oracle(16)
    rng = np.random.default_rng(3)
    tau = rng.standard_normal((16 ** 3, 6))
    F = LO.tau_force(co, tau)
    assert co.divergence(*F) < 1e-20 + 1e-12 * co.energy(*F, 1)
    # an isotropic stress (pressure-like) gives no force
    iso = np.zeros_like(tau)
    iso[:, :3] = rng.standard_normal((16 ** 3, 1))
    F0 = LO.tau_force(co, iso)
    assert max(np.max(np.abs(x)) for x in F0) < 1e-10


def test_vcorrect_sets_mode_energy_and_keeps_helicity():
    """vcorrect (heli = 0) gives every correctable mode the energy
    E = |v|^2 + 2 tepq dt ef / eold, keeps the helicity of the field and
    leaves it solenoidal."""
    o = Oracle(32)
    o.set_kmax(100.0)
    v, _ = o.random_solenoidal(8, 1.0, 10.0, 0, 1.0)
    _, _, _, kn2, kk2 = o.tables()
    s = np.where(kk2 > 0, kk2, 1.0) ** (-11.0 / 12.0)
    v = [x * s for x in v]
    Ek, _ = o.spectrumc(*v, 1, 0)
    tepq, _, _ = o.evedqnm(Ek, 1e-3, 2.0)
    n6 = float(32 ** 6)
    ef = (np.abs(v[0]) ** 2 + np.abs(v[1]) ** 2 + np.abs(v[2]) ** 2) / n6
    dt = 0.01
    vc = o.vcorrect(v, ef, tepq, Ek, dt)
    e_new = (np.abs(vc[0]) ** 2 + np.abs(vc[1]) ** 2 + np.abs(vc[2]) ** 2) / n6
    km = np.clip((np.sqrt(kk2) + np.float32(0.501)).astype(int) - 1, 0, len(Ek) - 1)
    mask = (kn2 <= o.kmax) & (kk2 > 0)
    target = ef + 2 * tepq[km] * dt * ef / Ek[km]
    hit = np.abs(e_new[mask] / target[mask] - 1) < 1e-9
    assert hit.mean() > 0.99
    assert abs(o.helicity(*vc) - o.helicity(*v)) < 1e-12 * abs(o.helicity(*v))
    assert o.divergence(*vc) < 1e-28
    assert not any(np.isnan(x).any() for x in vc)


# ------------------------------------------------- helical EDQNM (heli = 1)
def test_helical_evedqnm_branches():
    """evedqnm with hel = 1 (pseudospec3D_edqnm.f90:72-83): a helicity
    spectrum that cannot be fitted (zero) leaves cusp in charge, so the
    helicity transfer and diffusivity vanish; a maximally helical-leaning
    H(k) = a k E(k) takes full_cusp, whose eddy viscosity is positive over
    the resolved shells and whose helicity terms are non-zero."""
    n, kc = 128, 42
    o = Oracle(n)
    o.set_kmax(float(kc * kc))
    E = kolmogorov(n, kc)
    tepq, thpq, tve, tvh, Ext, Hxt = o.evedqnm_h(E, np.zeros_like(E), 1e-4, 10.0, hel=1)
    assert np.all(thpq == 0) and np.all(tvh == 0)
    assert np.all(tve[:kc] > 0)
    H = 0.3 * np.arange(1, n // 2 + 2) * E
    tepq, thpq, tve, tvh, Ext, Hxt = o.evedqnm_h(E, H, 1e-4, 10.0, hel=1)
    assert np.all(tve[:kc] > 0) and np.all(tve[kc:] == 0)
    assert np.any(tvh[:kc] != 0) and np.any(thpq[:kc] != 0)
    # full_cusp works on the halved extrapolations (:212-215)
    assert np.all(Ext[kc:3 * kc] > 0) and np.all(Hxt[kc:3 * kc] > 0)
    # hel = 0 through the helical entry point equals the plain evedqnm
    t0, _, v0, h0, x0, _ = o.evedqnm_h(E, H, 1e-4, 10.0, hel=0)
    t1, v1, x1 = o.evedqnm(E, 1e-4, 10.0)
    assert np.array_equal(t0, t1) and np.array_equal(v0, v1) and np.array_equal(x0, x1) and np.all(h0 == 0)


def test_helical_edqnm_run_reduces_to_the_plain_run_without_helicity_flag():
    """The heli-aware step with hel = 0 is the heli = 0 step bit for bit;
    with hel = 1 the run stays finite, solenoidal and different."""
    n, kc = 32, 10
    o = Oracle(n)
    o.set_kmax(float(kc * kc))
    v0, _ = o.random_solenoidal(7, 1.0, 10.0, 1, 1.0)
    f, _ = o.random_solenoidal(8, 2.0, 3.0, 0, 1.0)
    a = o.edqnm_run(3, 2, 2e-3, 1e-3, v0, f, t0=0.5)
    b = o.edqnm_run(3, 2, 2e-3, 1e-3, v0, f, t0=0.5, hel=0)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    lib = o.lib
    c = [x.copy() for x in v0]
    lib.o_edqnm_run_h(o.h, 3, 2, 2e-3, 1e-3, 1.4, 0.5, 1, 0, *[x.ctypes.data for x in c],
                      *[x.ctypes.data for x in f])
    assert all(np.array_equal(x, y) for x, y in zip(a, c))
    d = o.edqnm_run(3, 2, 2e-3, 1e-3, v0, f, t0=0.5, hel=1)
    assert all(np.all(np.isfinite(x)) for x in d)
    assert o.divergence(*d) < 1e-20 * max(1.0, o.energy(*d, 1))
    assert rel_l2(d, a) > 0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_library_helical_evedqnm_matches_oracle(prec):
    """ghost_evedqnm_hel (host) against the oracle's evedqnm with hel = 1,
    on a spectrum pair that takes full_cusp and on one that falls back to cusp."""
    from ghost_b200.les import evedqnm_hel
    n, kc = 128, 42
    o = Oracle(n, precision=prec)
    o.set_kmax(float(kc * kc))
    E = kolmogorov(n, kc)
    tol = 1e-12 if prec == "fp64" else 1e-5
    for H in (0.3 * np.arange(1, n // 2 + 2) * E, np.zeros_like(E)):
        for t in (0.5, 5.0):
            ref = o.evedqnm_h(E, H, 1e-3, t, hel=1)
            got = evedqnm_hel(n, float(kc * kc), E, H, 1e-3, t, hel=1, precision=prec)
            for a, b in zip(got, ref):
                assert rel_l2(a, b) <= tol


def test_helical_projection_has_one_sign_of_helicity():
    o = Oracle(32)
    v, _ = o.random_solenoidal(3, 1.0, 10.0, 1, 1.0)
    h = LO.helical(o, v, +1)
    _, Hk = o.spectrumc(*h, 1, 1)
    Ek, _ = o.spectrumc(*h, 1, 0)
    kk = np.arange(1, len(Hk) + 1)
    live = Ek > 1e-20
    # maximal helicity: H(k) = k E(k) in spectrumc's normalisation (up to shell rounding)
    assert np.all(Hk[live] > 0) and np.allclose(Hk[live], kk[live] * Ek[live], rtol=0.3)
    assert o.divergence(*h) < 1e-20
