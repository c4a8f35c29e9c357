"""The LES kernels (ghost_les_*) against the oracle: sharp truncation,
training samples (gradients and subgrid stresses), the closure forces
(EDQNM eddy viscosity, the MLP stress divergence and the MLP spectral eddy
viscosity), the EDQNM LES run,
and that the closure-free LES is the plain HD run.

Tolerances: FP64 1e-12 (single passes) to 1e-10 (runs of several steps),
1e-7 for the float32 sample arrays; FP32 1e-5; the MLP closure 2e-2 (BF16 network against the oracle network
with the same BF16 rounding, where accumulation order flips some roundings)."""
import numpy as np
import pytest

from oracle import les_oracle as LO
from oracle import mlp_oracle as M
from oracle.oracle import Oracle
from tests.conftest import rel_l2
from tests.helpers import rand_spectral, to_dev, to_host

pytestmark = pytest.mark.gpu


def kolmogorov_field(o, seed, kc):
    """A solenoidal field with E(k) ~ k^-5/3 on 1 <= |k| <= kc."""
    v, _ = o.random_solenoidal(seed, 1.0, float(kc), 0, 1.0)
    _, _, _, _, kk2 = o.tables()
    s = np.where(kk2 > 0, kk2, 1.0) ** (-11.0 / 12.0)
    return [(x * s).astype(o.cdt) for x in v]


def setup(prec, N=64, n=32, kc=10):
    from ghost_b200 import Ghost
    from ghost_b200.les import LES
    fo, co = Oracle(N, precision=prec), Oracle(n, precision=prec)
    co.set_kmax(float(kc * kc))
    gf, gc = Ghost(N, precision=prec), Ghost(n, precision=prec)
    return fo, co, gf, gc, LES(gc, kc)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_truncate(prec):
    fo, co, gf, gc, les = setup(prec)
    a = rand_spectral(fo, 1)
    out = to_host(les.truncate(gf, to_dev(a)))
    ref = fo.les_truncate(co, a, 10)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_samples(prec):
    fo, co, gf, gc, les = setup(prec)
    fo64, co64 = Oracle(64), Oracle(32)
    v = kolmogorov_field(fo64, 3, 21)
    cd = gf.cdtype_np
    x, tau = les.samples(gf, *[to_dev(a.astype(cd)) for a in v], 1.0)
    rx, rt = LO.samples(fo64, co64, [a.astype(cd).astype(np.complex128) for a in v], 10)
    # x and tau are float32 arrays (the network's input format): the FP64
    # path is exact up to that final rounding
    tol = 1e-7 if prec == "fp64" else 2e-5
    assert rel_l2(to_host(x), rx) <= tol
    assert rel_l2(to_host(tau), rt) <= tol


def test_features_and_tau_force():
    fo, co, gf, gc, les = setup("fp64")
    v = kolmogorov_field(co, 4, 10)
    x = les.features(*[to_dev(a) for a in v], 0.5, 2.0)
    assert rel_l2(to_host(x), LO.features(co, v, 0.5, 2.0)) <= 1e-7  # float32 output
    tau = np.random.default_rng(5).standard_normal((32 ** 3, 6)).astype(np.float32)
    f = [rand_spectral(co, 6 + a) for a in range(3)]
    F = les.tau_force(to_dev(tau), 0.25, [to_dev(a) for a in f])
    ref = LO.tau_force(co, tau.astype(np.float64), 0.25, f)
    assert rel_l2([to_host(a) for a in F], ref) <= 1e-12


def test_edqnm_closure_force():
    fo, co, gf, gc, les = setup("fp64")
    v = kolmogorov_field(co, 8, 10)
    les.set_model("edqnm", kolmo=1.4)
    les.set_time(2.0)
    F = les.closure_force(1e-3, *[to_dev(a) for a in v])
    Ek, _ = co.spectrumc(*v, 1, 0)
    _, tve, _ = co.evedqnm(Ek, 1e-3, 2.0)
    assert np.max(tve) > 0
    tve_g, _, Ek_g = les.edqnm_last()
    assert rel_l2(Ek_g, Ek) <= 1e-13
    assert rel_l2(tve_g, tve) <= 1e-12
    assert rel_l2([to_host(a) for a in F], LO.eddy_force(co, v, tve)) <= 1e-12


def test_edqnm_les_run():
    fo, co, gf, gc, les = setup("fp64")
    v = kolmogorov_field(co, 9, 10)
    f, _ = co.random_solenoidal(10, 2.0, 3.0, 0, 1.0)
    les.set_model("edqnm")
    les.set_time(1.0)
    V = [to_dev(a) for a in v]
    les.run(3, 2, 1e-3, 1e-3, *V, *[to_dev(a) for a in f])
    ref = co.edqnm_run(3, 2, 1e-3, 1e-3, v, f, t0=1.0)
    assert rel_l2([to_host(a) for a in V], ref) <= 1e-11


def test_helical_edqnm_closure_force():
    """heli = 1 on a maximally helical field: the helicity spectrum joins
    the fit, full_cusp gives tvh and thpq, and the force adds tvh(k) curl v."""
    fo, co, gf, gc, les = setup("fp64")
    v = LO.helical(co, kolmogorov_field(co, 8, 10), +1)
    les.set_model("edqnm", kolmo=1.4)
    les.set_helicity(1)
    les.set_time(2.0)
    F = les.closure_force(1e-3, *[to_dev(a) for a in v])
    Ek, Hk = co.spectrumc(*v, 1, 1)
    tepq, thpq, tve, tvh, _, _ = co.evedqnm_h(Ek, Hk, 1e-3, 2.0, hel=1)
    assert np.max(tve) > 0 and np.any(tvh != 0) and np.any(thpq != 0)  # full_cusp ran
    tve_g, tepq_g, Ek_g = les.edqnm_last()
    tvh_g, thpq_g, Hk_g = les.edqnm_last_hel()
    assert rel_l2(Hk_g, Hk) <= 1e-13
    for a, b in ((tve_g, tve), (tepq_g, tepq), (tvh_g, tvh), (thpq_g, thpq)):
        assert rel_l2(a, b) <= 1e-12
    assert rel_l2([to_host(a) for a in F], LO.eddy_force(co, v, tve, tvh=tvh)) <= 1e-12


@pytest.mark.parametrize("shape_seed", [12, 13])
def test_helical_edqnm_les_run(shape_seed):
    """Three RK2 steps of the LES with GHOST's helical EDQNM closure
    (full_cusp, the tvh curl v term, vcorrect's helicity target) against the
    oracle's restatement of edqnmhd_rkstep2 with heli = 1."""
    fo, co, gf, gc, les = setup("fp64")
    # positive helicity in every shell but away from the maximal limit, where
    # vcorrect's sqrt(1 - H^2 / (k^2 E^2 / 4)) vanishes and rounding dominates
    u = kolmogorov_field(co, shape_seed, 10)
    v = [a + 0.4 * b for a, b in zip(LO.helical(co, u, +1), LO.helical(co, u, -1))]
    _, Hk = co.spectrumc(*v, 1, 1)
    assert np.all(Hk[:10] > 0)
    f, _ = co.random_solenoidal(10, 2.0, 3.0, 0, 1.0)
    f = LO.helical(co, f, +1)
    les.set_model("edqnm")
    les.set_helicity(1)
    les.set_time(1.0)
    V = [to_dev(a) for a in v]
    les.run(3, 2, 1e-3, 1e-3, *V, *[to_dev(a) for a in f])
    ref = co.edqnm_run(3, 2, 1e-3, 1e-3, v, f, t0=1.0, hel=1)
    assert rel_l2([to_host(a) for a in V], ref) <= 1e-11
    # the helical closure changed the run
    plain = co.edqnm_run(3, 2, 1e-3, 1e-3, v, f, t0=1.0, hel=0)
    assert rel_l2(ref, plain) > 1e-9


def test_mlp_closure_force():
    from ghost_b200.les import MLP
    fo, co, gf, gc, les = setup("fp32")
    v = kolmogorov_field(co, 11, 10)
    p = M.glorot(12)
    m = MLP(0)
    m.params = p
    les.set_model("mlp", m, grad_scale=0.3, tau_scale=0.05, delta=1.0)
    F = les.closure_force(1e-3, *[to_dev(a) for a in v])
    co64 = Oracle(32)
    co64.set_kmax(100.0)
    v64 = [a.astype(np.complex128) for a in v]
    x = LO.features(co64, v64, 0.3, 1.0).astype(np.float32)
    y = M.forward(p, x, emulate=True).astype(np.float64)
    ref = LO.tau_force(co64, y, 0.05)
    assert rel_l2([to_host(a).astype(np.complex128) for a in F], ref) <= 2e-2


def test_spectral_features():
    import torch
    fo, co, gf, gc, les = setup("fp64")
    v = kolmogorov_field(co, 21, 10)
    Ek, _ = co.spectrumc(*v, 1, 0)
    x = les.spectral_features(torch.tensor(Ek, device="cuda"))
    ref = LO.spectral_features(Ek, 10)
    assert x.shape == (10, 10)
    assert rel_l2(to_host(x), ref) <= 1e-7  # float32 output
    assert np.all(ref[:, 8:] == 0) and ref[-1, 6] == 1.0


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_spectral_closure_force(prec):
    """The spectral closure: device spectrum -> shell inputs -> network ->
    tve -> eddy-viscous force, against the oracle's eddy force with the tve
    of the same chain (exact up to the force's arithmetic), and against the
    oracle network (BF16 emulated) end to end."""
    import torch
    from ghost_b200.les import MLP
    fo, co, gf, gc, les = setup(prec)
    v = kolmogorov_field(co, 22, 10)
    f = [rand_spectral(co, 23 + a) for a in range(3)]
    p = M.glorot(24)
    m = MLP(0)
    m.params = p
    V = [to_dev(a) for a in v]
    Eg, _ = gc.spectrumc(*V, 1, 0)
    yg = to_host(m.forward(les.spectral_features(torch.tensor(Eg, device="cuda"))))
    # the sign that makes most of this random network's eddy viscosities positive
    # (the rest are clamped at zero)
    scale = 0.02 if np.count_nonzero(yg[:, 0] > 0) >= 5 else -0.02
    les.set_model("mlp_spectral", m, tau_scale=scale)
    F = les.closure_force(1e-3, *V, [to_dev(a) for a in f])
    # the closure holds tau_scale as a float
    tve = LO.spectral_tve(yg[:, 0], Eg, 10, 17, float(np.float32(scale)))
    assert np.count_nonzero(tve) >= 5 and np.all(tve >= 0)
    tol = 1e-12 if prec == "fp64" else 1e-5
    ref = LO.eddy_force(co, v, tve, f)
    assert rel_l2([to_host(a) for a in F], ref) <= tol
    # end to end against the oracle's spectrum, inputs and network
    co64 = Oracle(32)
    co64.set_kmax(100.0)
    v64 = [a.astype(np.complex128) for a in v]
    E64, _ = co64.spectrumc(*v64, 1, 0)
    y64 = M.forward(p, LO.spectral_features(E64, 10), emulate=True).astype(np.float64)
    tve64 = LO.spectral_tve(y64[:, 0], E64, 10, 17, scale)
    ref64 = LO.eddy_force(co64, v64, tve64, [a.astype(np.complex128) for a in f])
    assert rel_l2([to_host(a).astype(np.complex128) for a in F], ref64) <= 2e-2


def test_spectral_closure_arguments():
    from ghost_b200 import Ghost
    from ghost_b200._lib import GhostError
    from ghost_b200.les import LES, MLP
    fo, co, gf, gc, les = setup("fp32")
    with pytest.raises(GhostError):
        les.set_model("mlp_spectral")  # no network
    g3 = Ghost(32, precision="fp32")
    with pytest.raises(GhostError):
        LES(g3, 3).set_model("mlp_spectral", MLP(0))  # fewer than 4 shells


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_les_without_closure_is_hd_run(prec):
    from ghost_b200 import Ghost
    fo, co, gf, gc, les = setup(prec)
    v = kolmogorov_field(co, 13, 10)
    f, _ = co.random_solenoidal(14, 2.0, 3.0, 0, 1.0)
    A = [to_dev(a) for a in v]
    B = [to_dev(a) for a in v]
    F = [to_dev(a) for a in f]
    les.run(4, 4, 1e-3, 1e-3, *A, *F)
    g2 = Ghost(32, precision=prec)
    g2.lib.ghost_ctx_set_kmax(g2.h, 100.0)
    g2.hd_run(4, 4, 1e-3, 1e-3, *B, *F)
    for a, b in zip(A, B):
        assert np.array_equal(to_host(a), to_host(b))


def _mlp_les(prec, p, fallback):
    from ghost_b200.les import MLP
    fo, co, gf, gc, les = setup(prec)
    m = MLP(0)
    m.params = p
    les.set_model("mlp", m, grad_scale=0.3, tau_scale=0.05, delta=1.0, kolmo=1.4)
    les.set_time(1.0)
    if fallback:
        les.set_fallback(True, 10.0)
    return co, les, m


def test_mlp_fallback_to_edqnm():
    """A network whose stresses overflow makes the first step non-finite: the
    step is redone with EDQNM, which then matches an EDQNM-only run exactly."""
    p = M.glorot(12) * np.float32(1e30)
    co, les, m = _mlp_les("fp32", p, True)
    v = kolmogorov_field(co, 15, 10)
    f, _ = co.random_solenoidal(16, 2.0, 3.0, 0, 1.0)
    A = [to_dev(a) for a in v]
    F = [to_dev(a) for a in f]
    les.run(3, 2, 1e-3, 1e-3, *A, *F)
    assert les.status() == ("edqnm", 0)
    _, _, _, _, ref = setup("fp32")
    ref.set_model("edqnm", kolmo=1.4)
    ref.set_time(1.0)
    B = [to_dev(a) for a in v]
    ref.run(3, 2, 1e-3, 1e-3, *B, *F)
    for a, b in zip(A, B):
        h = to_host(a)
        assert np.all(np.isfinite(h))
        assert np.array_equal(h, to_host(b))
    # without the fallback the same network leaves a non-finite field
    _, les2, m2 = _mlp_les("fp32", p, False)
    C = [to_dev(a) for a in v]
    les2.run(1, 2, 1e-3, 1e-3, *C, *F)
    assert not all(np.all(np.isfinite(to_host(a))) for a in C)
    assert les2.status() == ("mlp", -1)


def test_mlp_fallback_idle_on_a_sane_network():
    """With a working network the guarded run is the unguarded one, bit for bit."""
    p = M.glorot(12)
    co, les, m = _mlp_les("fp32", p, True)
    _, les2, m2 = _mlp_les("fp32", p, False)
    v = kolmogorov_field(co, 17, 10)
    A = [to_dev(a) for a in v]
    B = [to_dev(a) for a in v]
    les.run(3, 2, 1e-3, 1e-3, *A)
    les2.run(3, 2, 1e-3, 1e-3, *B)
    assert les.status() == ("mlp", -1)
    for a, b in zip(A, B):
        assert np.array_equal(to_host(a), to_host(b))
