"""The oracle's HD operators and RK step against analytic known answers taken
from the reference's own example initial conditions and consistency checks."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_l2
from tests.helpers import solenoidal_ic


def test_wavenumber_tables_follow_main3d():
    # main3D.fpp:1746-1749: kx(i)=i-1 for i<=n/2, kx(i+n/2)=i-n/2-1
    o = Oracle(16)
    kx, ky, kz, kn2, kk2 = o.tables()
    assert kx.tolist() == [0, 1, 2, 3, 4, 5, 6, 7, -8, -7, -6, -5, -4, -3, -2, -1]
    assert o.kmax == pytest.approx(16 * 16 / 9.0)
    assert o.tiny == pytest.approx(min(1e-5, 0.1 / 16**2))
    assert kn2[3, 2, 1] == 9 + 4 + 1 and np.shares_memory is not None
    # anisotropic ARBSIZE box: kn2 normalised per axis, kk2 physical
    a = Oracle(32, 32, 8, Lx=1, Ly=1, Lz=0.25, arbsize=True)
    kx, ky, kz, kn2, kk2 = a.tables()
    assert a.anis == 1 and a.kmax == pytest.approx(1 / 9.0)
    assert kz[1] == 4.0 and a.nmax == 32
    assert kk2[1, 0, 1] == pytest.approx(1 + 16)
    assert kn2[1, 0, 1] == pytest.approx(1 / 32**2 + 1 / 8**2)


def test_randu_sequence_is_park_miller_with_mask():
    import ctypes
    o = Oracle(16)
    s = ctypes.c_int32(1000)
    seq = [o.lib.o_randu(ctypes.byref(s)) for _ in range(4)]
    # recompute the masked Park-Miller sequence independently
    idum, out = 1000, []
    for _ in range(4):
        idum ^= 123459876
        k = idum // 127773
        idum = 16807 * (idum - k * 127773) - 2836 * k
        if idum < 0:
            idum += 2147483647
        out.append((idum * 2.0**-31 - 0.5) * 2)
        idum ^= 123459876
    assert np.allclose(seq, out, rtol=0, atol=1e-15)
    assert s.value == idum


def test_abc_beltrami_flow_decays_exactly():
    """examples/initialv.f90_abc with kdn=kup=1 is a Beltrami flow: curl v = v,
    the projected nonlinear term vanishes and E(t) = E0 exp(-2 nu t)."""
    o = Oracle(32)
    R = o.abc(1, 1, 1.0, 1.0, 1.0)
    v = [o.fftp3d_real_to_complex(x) for x in R]
    v = list(o.normalize(*v, 1.0))
    nl = o.prodre3(*v)
    g = [o.nonlhd3(*nl, d) for d in (1, 2, 3)]
    vmax = max(np.abs(x).max() for x in v)
    assert max(np.abs(x).max() for x in g) < 1e-13 * vmax
    nu, dt, n = 0.01, 1e-3, 50
    E0 = o.energy(*v, 1)
    v2 = o.hd_run(n, 4, dt, nu, v)
    assert o.energy(*v2, 1) / E0 == pytest.approx(np.exp(-2 * nu * n * dt), rel=1e-12)


def test_solenoidal_ic_properties():
    o = Oracle(32)
    v = solenoidal_ic(o)
    assert o.energy(*v, 1) == pytest.approx(1.0, rel=1e-13)
    assert o.divergence(*v) < 1e-28
    # Hermitian kx=0 plane: v(0,-ky,-kz) = conj v(0,ky,kz)
    p = v[0][0]
    flip = np.roll(p[::-1, ::-1], 1, axis=(0, 1))
    assert np.abs(p - np.conj(flip)).max() < 1e-15
    Ek, _ = o.spectrumc(*v, 1, 0)
    assert int(np.argmax(Ek)) + 1 == 2  # E(k) ~ k^4 exp(-k^2/2) peaks at k=2


def test_energy_budget_matches_reference_consistency_check():
    """3D/src/README:490-502: without random forcing dE/dt = -2 nu Omega + eps,
    with E = <v^2>/2, Omega = <w^2>/2 (balance.txt columns 2-4)."""
    o = Oracle(32)
    v = solenoidal_ic(o, seed=7)
    f, _ = o.random_solenoidal(11, 2.0, 3.0, 0, 1.0)
    nu, dt = 2e-3, 1e-4
    e = []
    vv = v
    for _ in range(3):
        e.append((o.energy(*vv, 1), o.energy(*vv, 0), o.cross(*vv, *f, 1)))
        vv = o.hd_run(1, 4, dt, nu, vv, f)
    e.append((o.energy(*vv, 1), o.energy(*vv, 0), o.cross(*vv, *f, 1)))
    dEdt = (e[2][0] - e[0][0]) / 2 / (2 * dt)  # <v^2>/2 centred difference
    rhs = -nu * e[1][1] + e[1][2]             # -2 nu Omega + eps, Omega=<w^2>/2
    assert dEdt == pytest.approx(rhs, rel=1e-4)


def test_nonlinear_term_is_solenoidal_and_divergence_free_update():
    o = Oracle(32)
    v = solenoidal_ic(o, seed=3)
    nl = o.prodre3(*v)
    g = [o.nonlhd3(*nl, d) for d in (1, 2, 3)]
    assert o.divergence(*g) < 1e-24 * o.energy(*g, 1) + 1e-30
    v2 = o.hd_run(2, 2, 1e-3, 2e-3, v)
    assert o.divergence(*v2) < 1e-28


def test_rk_truncation_zeroes_mean_and_dealiased_modes():
    o = Oracle(16)
    v = solenoidal_ic(o, seed=5)
    v = [x + 1e-3 for x in v]  # pollute every mode
    C = [x.copy() for x in v]
    f = [np.zeros_like(x) for x in v]
    out = o.hd_rkstep2(2, 1e-3, 1e-3, v, C, f)
    kx, ky, kz, kn2, kk2 = o.tables()
    mask = (kn2 <= o.kmax) & (kn2 >= o.tiny)
    for x in out:
        assert np.all(x[~mask] == 0)
        assert x[0, 0, 0] == 0


def test_fp32_oracle_tracks_fp64():
    o64, o32 = Oracle(32), Oracle(32, precision="fp32")
    v = solenoidal_ic(o64)
    a = o64.hd_run(5, 2, 1e-3, 2e-3, v)
    b = o32.hd_run(5, 2, 1e-3, 2e-3, [x.astype(np.complex64) for x in v])
    assert rel_l2(b, a) < 1e-5


def test_spectrum_sums_to_energy():
    o = Oracle(32)
    v = solenoidal_ic(o)
    Ek, Hk = o.spectrumc(*v, 1, 1)
    # shells beyond nmax/2+1 are dropped; the IC lives below N/3
    assert Ek.sum() == pytest.approx(o.energy(*v, 1), rel=1e-12)
    assert Hk.sum() == pytest.approx(o.helicity(*v), rel=1e-10, abs=1e-14)


def test_transfer_spectra_identities():
    """entrans / heltrans (pseudospec3D_hd.f90:1629-1949) on the oracle:
    the nonlinear term moves energy and helicity between shells without
    creating either (v.(w x v) = w.(w x v) = 0 at every grid point, so the
    shell sums add up to zero), entrans of a field with itself is its
    kinetic spectrum, and with kin = 0 its curl spectrum (solenoidal v)."""
    o = Oracle(32)
    v = solenoidal_ic(o, seed=7)
    nl = o.prodre3(*v)
    T = o.entrans(*v, *nl, kin=1)
    H = o.heltrans(*v, *nl)
    Ek, _ = o.spectrumc(*v, 1, 0)
    Wk, _ = o.spectrumc(*v, 0, 0)
    assert abs(T.sum()) <= 1e-12 * np.abs(T).sum()
    assert abs(H.sum()) <= 1e-12 * np.abs(H).sum()
    assert np.abs(T).sum() > 0 and np.abs(H).sum() > 0
    assert rel_l2(o.entrans(*v, *v, kin=1), Ek) <= 1e-14
    assert rel_l2(o.entrans(*v, *v, kin=0), Wk) <= 1e-12


@pytest.mark.parametrize("box", [dict(), dict(Lx=1.0, Ly=1.0, Lz=0.5, arbsize=True)])
def test_anisotropic_spectra_identities(box):
    """specpara / specperp and the binned transfers (pseudospec3D_rot.f90)
    on the oracle: for a truncated zero-mean field every mode lands in a
    bin, so each anisotropic spectrum sums to its shell-spectrum total;
    specpara's total is its horizontal plus vertical sums, bin by bin, and
    specperp's horizontal and vertical sums are the kz = 0 plane's share."""
    o = Oracle(32, 32, 16, **box)
    v = solenoidal_ic(o, seed=9)
    nl = o.prodre3(*v)
    Ek, _ = o.spectrumc(*v, 1, 0)
    _, Hk = o.spectrumc(*v, 1, 1)
    for mode in (0, 1):
        E, H = o.spec_aniso(mode, *v, kin=1, hel=1)
        assert abs(E[0].sum() - Ek.sum()) <= 1e-13 * Ek.sum()
        assert abs(H[0].sum() - Hk.sum()) <= 1e-12 * np.abs(Hk).sum()
        if mode == 0:
            assert np.allclose(E[0], E[1] + E[2], rtol=1e-14, atol=0)
        else:
            assert (E[1] + E[2]).sum() <= E[0].sum()
        T = o.entrans(*v, *nl, kin=1)
        Ta = o.trans_aniso(mode, *v, *nl, kin=1)
        assert abs(Ta.sum() - T.sum()) <= 1e-12 * np.abs(T).sum()
        Hta = o.trans_aniso(mode, *v, *nl, curl=True)
        assert abs(Hta.sum() - o.heltrans(*v, *nl).sum()) <= 1e-12 * np.abs(Hta).sum()


def test_havgcomp_profiles_identities():
    """havgcomp (pseudospec3D_bouss.f90:19-554) on the oracle: the z-means
    of the horizontal kinetic profiles add up to <|v|^2>, the z-mean of
    <w s> is the cross term <w s>, and type 9 repeats type 0 as in GHOST."""
    o = Oracle(32, 32, 16, Lx=1.0, Ly=1.0, Lz=0.5, arbsize=True)
    v = solenoidal_ic(o, seed=11)
    s = o.random_solenoidal(12, 1.0, 4.0, 0, 1.0)[0][0]
    z = np.zeros_like(s)
    h3 = o.havgcomp(*v, s, 1.0, 8.0, 3)
    h4 = o.havgcomp(*v, s, 1.0, 8.0, 4)
    assert abs((h3 + h4).mean() - o.energy(*v, 1)) <= 1e-12 * o.energy(*v, 1)
    h10 = o.havgcomp(*v, s, 1.0, 8.0, 10)
    ws = o.cross(z, z, v[2], z, z, s, 1)
    assert abs(h10.mean() - ws) <= 1e-12 * max(abs(ws), 1e-30) + 1e-15
    assert np.array_equal(o.havgcomp(*v, s, 1.0, 8.0, 9), o.havgcomp(*v, s, 1.0, 8.0, 0))
    for t in range(11):
        assert np.all(np.isfinite(o.havgcomp(*v, s, 1.0, 8.0, t)))


def test_passive_scalar_identities():
    """The passive-scalar routines (pseudospec3D_phd.f90, phd_rkstep2.f90)
    on the oracle: the PHD step is the rotating Boussinesq step with no
    rotation, buoyancy or heat current; advection moves scalar variance
    between shells without creating it (sum of sctrans(th, -v.grad th) = 0);
    the scalar spectrum sums to the variance; variance(kin 0) weights by k^2."""
    o = Oracle(32, 32, 16, Lx=1.0, Ly=1.0, Lz=0.5, arbsize=True)
    v = solenoidal_ic(o, seed=21)
    th = o.random_solenoidal(22, 1.0, 4.0, 0, 1.0)[0][0]
    vp, thp = o.phd_run(2, 2, 1e-3, 1e-3, 2e-3, v, th)
    vb, thb = o.bouss_run(2, 2, 1e-3, 1e-3, 2e-3, 0.0, 0.0, 0.0, v, th)
    assert all(np.array_equal(a, b) for a, b in zip(vp, vb)) and np.array_equal(thp, thb)
    adv = o.advect3(*v, th)
    T = o.sctrans(th, adv)
    assert abs(T.sum()) <= 1e-12 * np.abs(T).sum()
    assert abs(o.spectrscc(th).sum() - o.variance(th, 1)) <= 1e-13 * o.variance(th, 1)
    assert o.variance(th, 0) > 0


def test_mhd_identities():
    """The MHD routines (pseudospec3D_mhd.f90, mhd_rkstep2.f90) on the
    oracle: v x v = 0; the gauged field is divergence-free; nonlin3 with no
    magnetic term is nonlhd3; with a = 0 the MHD run is the HD run."""
    o = Oracle(32)
    v = solenoidal_ic(o, seed=31)
    x = o.vector3(*v, *v)
    assert all(np.abs(q).max() <= 1e-14 * np.abs(v[0]).max() for q in x)
    w = [o.random_solenoidal(32 + q, 1.0, 6.0, 0, 1.0)[0][q] for q in range(3)]
    g = [o.gauge3(*w, d) for d in (1, 2, 3)]
    assert o.divergence(*g) <= 1e-20 * o.energy(*g, 1) + 1e-30
    z = [np.zeros_like(v[0]) for _ in range(3)]
    for d in (1, 2, 3):
        assert np.allclose(o.nonlin3(*w, *z, d), o.nonlhd3(*w, d), rtol=0, atol=1e-15 * np.abs(w[0]).max())
    vm, am = o.mhd_run(2, 2, 1e-3, 1e-3, 1e-3, v, z)
    vh = o.hd_run(2, 2, 1e-3, 1e-3, v)
    assert rel_l2(vm, vh) <= 1e-14
    assert all(np.abs(q).max() == 0 for q in am)


def test_phaseshift_keeps_energy_and_hermitian_plane():
    """phaseshift (pseudospec3D_hd.f90:2084-2148) with |cdump| = 1 on the
    oracle: the energy is unchanged, and a field that is Hermitian on the
    kx = 0 plane stays Hermitian there (mirror modes take conj(cdump))."""
    o = Oracle(16, 16, 32)
    v = solenoidal_ic(o, seed=51)
    cd = np.exp(0.7j)
    w = [o.phaseshift(x, cd) for x in v]
    assert abs(o.energy(*w, 1) - o.energy(*v, 1)) <= 1e-14 * o.energy(*v, 1)
    p0 = w[0][0]  # kx = 0 plane (ny, nz)
    ny, nz = p0.shape
    mirror = np.conj(p0[(-np.arange(ny)) % ny][:, (-np.arange(nz)) % nz])
    assert np.allclose(p0, mirror, rtol=0, atol=1e-14 * np.abs(p0).max())


def test_slowly_varying_forcing_interpolates():
    """rand = 2 (main3D.fpp:2646-2657): the forcing moves linearly from the
    old to the new random forcing over fstep steps and reaches it."""
    o = Oracle(16)
    a, _ = o.random_solenoidal(3, 2.0, 3.0, 0, 1.0)
    b, _ = o.random_solenoidal(4, 2.0, 3.0, 0, 1.0)
    fstep = 4
    for timef in range(fstep):
        f = o.forcing_slow(timef, fstep, a, b)
        w = np.float32(timef + 1) / np.float32(fstep)
        assert all(np.allclose(x, (1 - w) * p + w * q, rtol=0, atol=1e-15) for x, p, q in zip(f, a, b))
    last = o.forcing_slow(fstep - 1, fstep, a, b)
    assert all(np.array_equal(x, q) for x, q in zip(last, b))
