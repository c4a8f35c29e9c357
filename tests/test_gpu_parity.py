"""Parity of the CUDA library (through the C ABI) with the CPU oracle on the
same seeded inputs: transforms, spectral operators, reductions, initial
conditions and the fused RK substeps of the HD and Boussinesq solvers.

Tolerances: FP64 paths rel <= 1e-12 (1e-13 for single operators); the FP32
path against the FP64 oracle rel <= 1e-5."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_l2
from tests.helpers import rand_real, rand_spectral, solenoidal_ic, to_dev, to_host

pytestmark = pytest.mark.gpu


def ghost(*args, **kw):
    from ghost_b200 import Ghost
    return Ghost(*args, **kw)


GRIDS = [(16, 16, 16), (32, 64, 16), (64, 32, 128), (64, 64, 64)]


# ------------------------------------------------------------------ FFTs
@pytest.mark.parametrize("shape", GRIDS)
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fftp3d_real_to_complex(shape, prec):
    from ghost_b200 import GHOST_REAL_TO_COMPLEX
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    r = rand_real(o, 1)
    ref = o.fftp3d_real_to_complex(r)
    plan = g.fftp3d_create_plan(shape, GHOST_REAL_TO_COMPLEX)
    out = g.czeros()
    g.fftp3d_real_to_complex(plan, to_dev(r.astype(g.rdtype_np)), out)
    tol = 1e-13 if prec == "fp64" else 2e-6
    assert rel_l2(to_host(out), ref) < tol


@pytest.mark.parametrize("shape", GRIDS)
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fftp3d_complex_to_real(shape, prec):
    from ghost_b200 import GHOST_COMPLEX_TO_REAL
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    c = rand_spectral(o, 2)  # not Hermitian: exercises the kx=0 / Nyquist rule
    ref = o.fftp3d_complex_to_real(c)
    plan = g.fftp3d_create_plan(shape, GHOST_COMPLEX_TO_REAL)
    cin = to_dev(c.astype(g.cdtype_np))
    keep = cin.clone()
    out = g.rzeros()
    g.fftp3d_complex_to_real(plan, cin, out)
    tol = 1e-13 if prec == "fp64" else 2e-6
    assert rel_l2(to_host(out), ref) < tol
    assert bool((cin == keep).all())  # input left unmodified


def test_fft_host_arrays_equal_device_arrays():
    from ghost_b200 import GHOST_REAL_TO_COMPLEX
    o = Oracle(32)
    g = ghost(32)
    r = rand_real(o, 3)
    plan = g.fftp3d_create_plan((32, 32, 32), GHOST_REAL_TO_COMPLEX)
    host_out = np.zeros(o.sshape, np.complex128)
    g.fftp3d_real_to_complex(plan, r, host_out)
    dev_out = g.czeros()
    g.fftp3d_real_to_complex(plan, to_dev(r), dev_out)
    assert np.array_equal(host_out, to_host(dev_out))


def test_fft_round_trip_at_512_fp32():
    """Size-independent property at the benchmark size: c2r(r2c(x)) = N^3 x."""
    from ghost_b200 import GHOST_COMPLEX_TO_REAL, GHOST_REAL_TO_COMPLEX
    import torch
    n = 512
    g = ghost(n, precision="fp32")
    x = torch.randn((n, n, n), device="cuda", dtype=torch.float32, generator=torch.Generator("cuda").manual_seed(0))
    c = g.czeros()
    pf = g.fftp3d_create_plan((n, n, n), GHOST_REAL_TO_COMPLEX)
    pb = g.fftp3d_create_plan((n, n, n), GHOST_COMPLEX_TO_REAL)
    g.fftp3d_real_to_complex(pf, x, c)
    # Parseval: sum |x|^2 = (1/N^3) sum_k w_k |X_k|^2
    w = torch.full((c.shape[0], 1, 1), 2.0, device="cuda", dtype=torch.float64)
    w[0] = 1.0
    w[-1] = 1.0
    lhs = float((x.double() ** 2).sum())
    rhs = float((w * c.abs().double() ** 2).sum()) / n**3
    assert abs(lhs - rhs) / lhs < 1e-5
    y = g.rzeros()
    g.fftp3d_complex_to_real(pb, c, y)
    err = float((y / n**3 - x).norm() / x.norm())
    assert err < 1e-5


# ------------------------------------------------------------- operators
@pytest.fixture(scope="module")
def pair32():
    o = Oracle(32, 32, 64)
    g = ghost(32, 32, 64)
    a, b, c = (rand_spectral(o, s) for s in (11, 12, 13))
    return o, g, a, b, c


@pytest.mark.parametrize("dir", [1, 2, 3])
def test_derivk3_rotor3_nonlhd3(pair32, dir):
    o, g, a, b, c = pair32
    A, B, Cc = to_dev(a), to_dev(b), to_dev(c)
    out = g.czeros()
    g.derivk3(A, out, dir)
    assert rel_l2(to_host(out), o.derivk3(a, dir)) < 1e-15
    g.rotor3(A, B, out, dir)
    assert rel_l2(to_host(out), o.rotor3(a, b, dir)) < 1e-15
    g.nonlhd3(A, B, Cc, out, dir)
    assert rel_l2(to_host(out), o.nonlhd3(a, b, c, dir)) < 1e-15
    # output aliasing an input, as hd_rkstep2 does with nonlhd3(C4,C5,C6,C4,3)
    A2 = A.clone()
    g.nonlhd3(A2, B, Cc, A2, dir)
    assert rel_l2(to_host(A2), o.nonlhd3(a, b, c, dir)) < 1e-15


def test_laplak3_sharp(pair32):
    o, g, a, b, c = pair32
    A = to_dev(a)
    out = g.czeros()
    g.laplak3(A, out)
    assert rel_l2(to_host(out), o.laplak3(a)) < 1e-15
    g.sharp(A, out, np.pi / 7.0)
    assert np.array_equal(to_host(out), o.sharp(a, np.pi / 7.0))


def test_prodre3(pair32):
    o, g, a, b, c = pair32
    outs = [g.czeros() for _ in range(3)]
    g.prodre3(to_dev(a), to_dev(b), to_dev(c), *outs)
    ref = o.prodre3(a, b, c)
    assert rel_l2([to_host(x) for x in outs], list(ref)) < 1e-13


def test_reductions(pair32):
    o, g, a, b, c = pair32
    A, B, Cc = to_dev(a), to_dev(b), to_dev(c)
    for kin in (0, 1, 2):
        assert g.energy(A, B, Cc, kin) == pytest.approx(o.energy(a, b, c, kin), rel=1e-13)
    assert g.helicity(A, B, Cc) == pytest.approx(o.helicity(a, b, c), rel=1e-11, abs=1e-14)
    for kin in (0, 1):
        assert g.cross(A, B, Cc, B, Cc, A, kin) == pytest.approx(o.cross(a, b, c, b, c, a, kin), rel=1e-11)
    assert g.divergence(A, B, Cc) == pytest.approx(o.divergence(a, b, c), rel=1e-13)
    # deterministic: bit-identical on repeat
    assert g.energy(A, B, Cc, 0) == g.energy(A, B, Cc, 0)


@pytest.mark.parametrize("kin", [0, 1, 2])
def test_maxabs(kin):
    o = Oracle(32)
    g = ghost(32)
    v = solenoidal_ic(o, seed=21)
    got = g.maxabs(*[to_dev(x) for x in v], kin)
    assert got == pytest.approx(o.maxabs(*v, kin), rel=1e-13)


def test_spectrumc():
    o = Oracle(64)
    g = ghost(64)
    v = solenoidal_ic(o, seed=31)
    Ek, Hk = g.spectrumc(*[to_dev(x) for x in v], 1, 1)
    Ek0, Hk0 = o.spectrumc(*v, 1, 1)
    assert np.allclose(Ek, Ek0, rtol=1e-12, atol=1e-300)
    assert np.allclose(Hk, Hk0, rtol=1e-9, atol=1e-18)
    Ew, _ = g.spectrumc(*[to_dev(x) for x in v], 0, 0)
    Ew0, _ = o.spectrumc(*v, 0, 0)
    assert np.allclose(Ew, Ew0, rtol=1e-12, atol=1e-300)
    Ek2, _ = g.spectrumc(*[to_dev(x) for x in v], 1, 0)
    assert np.array_equal(Ek, Ek2)


def test_normalize_and_initial_condition():
    o = Oracle(64)
    g = ghost(64)
    v0 = solenoidal_ic(o, seed=1000)
    outs = [g.czeros() for _ in range(3)]
    seed = g.init_random_solenoidal(1000, 1.0, 64 / 3.0, 1, 1.0, *outs)
    _, seed0 = o.random_solenoidal(1000, 1.0, 64 / 3.0, 1, 1.0)
    assert seed == seed0
    assert rel_l2([to_host(x) for x in outs], v0) < 1e-14
    f0, _ = o.random_solenoidal(5, 2.0, 3.0, 0, 1.0)
    F = [to_dev(x * 3.0) for x in f0]
    g.normalize(*F, 1.0, 1)
    assert rel_l2([to_host(x) for x in F], f0) < 1e-14


# ------------------------------------------------------------ RK steps
def test_hd_cfg0_one_step_and_hundred_steps_fp64():
    """Config 0: 64^3 FP64, nu=2e-3, dt=1e-3, RK2, unit-energy seeded IC:
    rel L2 <= 1e-12 after one step and <= 1e-9 after 100 steps."""
    o = Oracle(64)
    g = ghost(64)
    v0 = solenoidal_ic(o, seed=1000)
    V = [to_dev(x) for x in v0]
    g.hd_run(1, 2, 1e-3, 2e-3, *V)
    ref1 = o.hd_run(1, 2, 1e-3, 2e-3, v0)
    assert rel_l2([to_host(x) for x in V], ref1) < 1e-12
    g.hd_run(99, 2, 1e-3, 2e-3, *V)
    ref100 = o.hd_run(99, 2, 1e-3, 2e-3, ref1)
    assert rel_l2([to_host(x) for x in V], ref100) < 1e-9


def test_hd_forced_rk4_fp64_and_fp32_against_fp64_oracle():
    """Config 1 at reduced size: forcing on 2<=|k|<=3 (f0=1), nu=1e-3,
    dt=5e-4, RK4; FP32 within 1e-5 of the FP64 oracle per step."""
    n = 64
    o = Oracle(n)
    v0 = solenoidal_ic(o, seed=1001)
    f, _ = o.random_solenoidal(2001, 2.0, 3.0, 0, 1.0)
    g64, g32 = ghost(n), ghost(n, precision="fp32")
    V64 = [to_dev(x) for x in v0]
    V32 = [to_dev(x.astype(np.complex64)) for x in v0]
    F64 = [to_dev(x) for x in f]
    F32 = [to_dev(x.astype(np.complex64)) for x in f]
    ref = v0
    for step in range(3):
        ref = o.hd_run(1, 4, 5e-4, 1e-3, ref, f)
        g64.hd_run(1, 4, 5e-4, 1e-3, *V64, *F64)
        g32.hd_run(1, 4, 5e-4, 1e-3, *V32, *F32)
        assert rel_l2([to_host(x) for x in V64], ref) < 1e-12
        assert rel_l2([to_host(x).astype(np.complex128) for x in V32], ref) < 1e-5
        # restart the FP32 run from the oracle state: per-step error
        V32 = [to_dev(x.astype(np.complex64)) for x in ref]


def test_rkstep1_rkstep2_equal_fused_run():
    o = Oracle(32)
    g = ghost(32)
    v0 = solenoidal_ic(o, seed=77)
    f, _ = o.random_solenoidal(78, 2.0, 3.0, 0, 1.0)
    A = [to_dev(x) for x in v0]
    B = [to_dev(x) for x in v0]
    F = [to_dev(x) for x in f]
    C = [g.czeros() for _ in range(3)]
    g.hd_rkstep1(*A, *C)
    for oo in (3, 2, 1):
        g.hd_rkstep2(oo, 1e-3, 1e-3, *A, *C, *F)
    g.hd_run(1, 3, 1e-3, 1e-3, *B, *F)
    assert all(bool((x == y).all()) for x, y in zip(A, B))
    ref = o.hd_run(1, 3, 1e-3, 1e-3, v0, f)
    assert rel_l2([to_host(x) for x in A], ref) < 1e-12


def test_hd_host_arrays_drop_in():
    """GHOST-style host arrays through the same entry points."""
    o = Oracle(32)
    g = ghost(32)
    v0 = solenoidal_ic(o, seed=9)
    V = [x.copy() for x in v0]
    g.hd_run(2, 2, 1e-3, 2e-3, *V)
    ref = o.hd_run(2, 2, 1e-3, 2e-3, v0)
    assert rel_l2(V, ref) < 1e-12


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_hd_host_arrays_move_live_rows_only(prec):
    """Host arrays move only the live box (the kx rows that hold kept modes,
    and in them the two blocks of y-lines that do) where that is exact: the
    forcing outside it is never read (garbage there changes nothing), and v
    comes back whole when it held nonzero values outside the box on the way
    in (they leave as zeros).  Every case against the same run on device
    arrays, bit for bit."""
    o = Oracle(32, precision=prec)
    g = ghost(32, precision=prec)
    v0 = solenoidal_ic(o, seed=21)
    f0, _ = o.random_solenoidal(22, 2.0, 3.0, 0, 1.0)
    live = 32 // 3 + 1  # kx rows 0..10 hold every mode with kn2 <= kmax at 32^3
    jt, jb = 11, 10      # and in them the y-lines ky = 0..10 and -10..-1, and the kz values 0..10, -10..-1
    zt, zb = (12, 10) if prec == "fp32" else (11, 10)  # the z blocks in whole 16-byte words
    rng = np.random.default_rng(23)
    junk = lambda x: (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)).astype(x.dtype)  # noqa: E731

    def device_run(v, f, nsteps=2):
        V = [to_dev(x) for x in v]
        g.hd_run(nsteps, 2, 1e-3, 2e-3, *V, *[to_dev(x) for x in f])
        return [to_host(x) for x in V]

    # 1: v zero beyond the live rows (every step's output), forcing with junk there
    v1 = device_run(v0, f0, 1)
    assert all(np.all(x[live:] == 0) and np.all(x[:, jt:32 - jb] == 0) and np.all(x[:, :, zt:32 - zb] == 0)
               for x in v1)
    f_junk = [x.copy() for x in f0]
    for x in f_junk:
        x[live:] = junk(x[live:])
        x[:live, jt:32 - jb] = junk(x[:live, jt:32 - jb])
        x[:live, :, zt:32 - zb] = junk(x[:live, :, zt:32 - zb])
    ref = device_run(v1, f0)
    V = [x.copy() for x in v1]
    g.hd_run(2, 2, 1e-3, 2e-3, *V, *[x.copy() for x in f_junk])
    assert all(np.array_equal(a, b) for a, b in zip(V, ref))
    # 2: v with nonzero values beyond the live rows: they are zero afterwards
    v2 = [x.copy() for x in v1]
    for x in v2:
        x[live + 2] = junk(x[live + 2])
    ref = device_run(v2, f0)
    V = [x.copy() for x in v2]
    g.hd_run(2, 2, 1e-3, 2e-3, *V, *[x.copy() for x in f0])
    assert all(np.array_equal(a, b) for a, b in zip(V, ref))
    assert all(np.all(x[live:] == 0) for x in V)
    # 2b: nonzero values in the middle y-lines of a live row only
    v2b = [x.copy() for x in v1]
    for x in v2b:
        x[0, 16] = junk(x[0, 16])
    ref = device_run(v2b, f0)
    V = [x.copy() for x in v2b]
    g.hd_run(2, 2, 1e-3, 2e-3, *V, *[x.copy() for x in f0])
    assert all(np.array_equal(a, b) for a, b in zip(V, ref))
    assert all(np.all(x[0, 16] == 0) for x in V)
    # 2c: nonzero values in the middle kz of a box line only
    v2c = [x.copy() for x in v1]
    for x in v2c:
        x[1, 2, 16] = 1.5 + 0.5j
    ref = device_run(v2c, f0)
    V = [x.copy() for x in v2c]
    g.hd_run(2, 2, 1e-3, 2e-3, *V, *[x.copy() for x in f0])
    assert all(np.array_equal(a, b) for a, b in zip(V, ref))
    assert all(x[1, 2, 16] == 0 for x in V)
    # 3: no step: v comes back as it went in, nonzero rows included
    V = [x.copy() for x in v2]
    g.hd_run(0, 2, 1e-3, 2e-3, *V, *[x.copy() for x in f0])
    assert all(np.array_equal(a, b) for a, b in zip(V, v2))


def test_hd_anisotropic_grid():
    o = Oracle(32, 16, 64)
    g = ghost(32, 16, 64)
    v0 = solenoidal_ic(o, seed=17)
    V = [to_dev(x) for x in v0]
    g.hd_run(3, 2, 1e-3, 2e-3, *V)
    ref = o.hd_run(3, 2, 1e-3, 2e-3, v0)
    assert rel_l2([to_host(x) for x in V], ref) < 1e-12


def test_abc_decay_on_gpu():
    o = Oracle(32)
    R = o.abc(1, 1, 1.0, 1.0, 1.0)
    v = list(o.normalize(*[o.fftp3d_real_to_complex(x) for x in R], 1.0))
    g = ghost(32)
    V = [to_dev(x) for x in v]
    E0 = g.energy(*V, 1)
    g.hd_run(50, 4, 1e-3, 0.01, *V)
    assert g.energy(*V, 1) / E0 == pytest.approx(np.exp(-2 * 0.01 * 0.05), rel=1e-12)


# ------------------------------------------------------------ Boussinesq
def test_advect3():
    o = Oracle(32, 32, 16, Lx=1, Ly=1, Lz=0.5, arbsize=True)
    g = ghost(32, 32, 16, Lx=1, Ly=1, Lz=0.5, arbsize=True)
    a, b, c, d = (rand_spectral(o, s, 1e-2) for s in (41, 42, 43, 44))
    out = g.czeros()
    g.advect3(*[to_dev(x) for x in (a, b, c, d)], out)
    assert rel_l2(to_host(out), o.advect3(a, b, c, d)) < 1e-13


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_bouss_steps(prec):
    """Config 2 physics on a small elongated ARBSIZE box (Lz = Lx/4)."""
    shape = (64, 64, 16)
    o = Oracle(*shape, Lx=1, Ly=1, Lz=0.25, arbsize=True)
    g = ghost(*shape, Lx=1, Ly=1, Lz=0.25, arbsize=True, precision=prec)
    v0, _ = o.random_solenoidal(55, 1.0, 6.0, 1, 1.0)
    th0 = rand_spectral(o, 56, 0.0)  # zero temperature perturbation
    args = (4, 2.5e-4, 5e-4, 5e-4, 0.5, 8.0, 8.0)
    ref_v, ref_th = o.bouss_run(2, *args, v0, th0)
    cd = g.cdtype_np
    V = [to_dev(x.astype(cd)) for x in v0]
    TH = to_dev(th0.astype(cd))
    g.bouss_run(2, *args, *V, TH)
    tol = 1e-12 if prec == "fp64" else 1e-5
    assert rel_l2([to_host(x).astype(np.complex128) for x in V] + [to_host(TH).astype(np.complex128)],
                  list(ref_v) + [ref_th]) < tol
    # buoyancy couples theta in after one step
    assert float(TH.abs().max()) > 0


def test_native_kernels_ran():
    g = ghost(32)
    n0 = g.launch_count()
    v = [g.czeros() for _ in range(3)]
    g.hd_run(1, 2, 1e-3, 1e-3, *v)
    assert g.launch_count() - n0 == 10  # 5 fused passes per substep


def test_bounded_wait_timeout_reports_and_recovers():
    """Failure detection without a fault: with the stall injected, every
    pipelined pass waits on a barrier nothing completes; after the (lowered)
    wait cap the kernels give up, drain their copies and return, the next
    synchronising call reports GHOST_ERR_TIMEOUT, and the context then works
    normally again."""
    from ghost_b200 import GhostError
    o = Oracle(64)
    g = ghost(64)
    v0 = solenoidal_ic(o, seed=3)
    V = [to_dev(x) for x in v0]
    g.set_wait_cap(1000)
    g.inject_stall(True)
    g.hd_run(1, 2, 1e-3, 2e-3, *V)
    with pytest.raises(GhostError) as err:
        g.synchronize()
    assert err.value.code == 5
    g.inject_stall(False)
    g.set_wait_cap(0)
    V = [to_dev(x) for x in v0]
    g.hd_run(1, 2, 1e-3, 2e-3, *V)
    g.synchronize()
    ref = o.hd_run(1, 2, 1e-3, 2e-3, v0)
    assert rel_l2([to_host(x) for x in V], ref) < 1e-12


def test_pruned_substeps_are_bitwise_equal_to_full_ones():
    """hd_run skips the known zeros outside the 2/3 truncation after its
    first substep; stepping with hd_rkstep2 (always full passes) must give
    the same bits."""
    o = Oracle(64)
    g = ghost(64, precision="fp32")
    v0 = [x.astype(np.complex64) for x in solenoidal_ic(o, seed=8)]
    A = [to_dev(x) for x in v0]
    B = [to_dev(x) for x in v0]
    C = [g.czeros() for _ in range(3)]
    g.hd_run(2, 2, 1e-3, 2e-3, *A)
    for _ in range(2):
        g.hd_rkstep1(*B, *C)
        for oo in (2, 1):
            g.hd_rkstep2(oo, 1e-3, 2e-3, *B, *C)
    assert all(bool((x == y).all()) for x, y in zip(A, B))


# ------------------------------------------------------ batches, ensembles
def test_batched_runs_match_independent_oracle_runs():
    """A batch of three 32^3 runs with their own seeds and viscosities, one
    launch per pass, against three oracle runs."""
    from ghost_b200 import Ghost
    o = Oracle(32)
    seeds, nus = [11, 12, 13], [5e-4, 2e-3, 5e-3]
    g = Ghost(32, precision="fp64", nruns=3)
    V = [g.czeros() for _ in range(3)]
    out_seeds = g.batch_init_random_solenoidal(seeds, 1.0, 32 / 3.0, 1, 1.0, *V)
    g.batch_set_nu(nus)
    g.hd_run(3, 2, 1e-3, 0.0, *V)
    nxh = 17
    for r in range(3):
        v0, s_after = o.random_solenoidal(seeds[r], 1.0, 32 / 3.0, 1, 1.0)
        assert out_seeds[r] == s_after
        ref = o.hd_run(3, 2, 1e-3, nus[r], v0)
        got = [to_host(x[r * nxh:(r + 1) * nxh]) for x in V]
        assert rel_l2(got, ref) < 1e-12
    e = g.batch_energy(*V, 1)
    assert np.allclose(e, [o.energy(*o.hd_run(3, 2, 1e-3, nus[r], o.random_solenoidal(seeds[r], 1.0, 32 / 3.0, 1, 1.0)[0]), 1)
                           for r in range(3)], rtol=1e-12)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_ensemble_graph_steps_match_oracle(prec):
    """Uneven classes (32^3 x 3, 64^3 x 2) stepped by the replayed CUDA graph
    after autotuning; every run against its own oracle run."""
    from ghost_b200 import Ensemble
    sizes, nruns = [32, 64], [3, 2]
    seeds = [101, 102, 103, 201, 202]
    nus = [5e-4, 1e-3, 5e-3, 8e-4, 3e-3]
    ens = Ensemble(sizes, nruns, precision=prec)
    ens.init(seeds, nus)
    cfg = ens.autotune(2, 1e-3)
    assert len(cfg) == 2 and all(c in (0, 1, 2, 3, 6, 7, 8, 14, 16, 22, 24, 30, 38, 46, 62, 126) for c in cfg)
    ens.run(4, 2, 1e-3)
    e = ens.energy(1)
    tol = 1e-12 if prec == "fp64" else 1e-5
    q = 0
    for c, (n, r) in enumerate(zip(sizes, nruns)):
        o = Oracle(n)
        fields = ens.fields(c)
        nxh = n // 2 + 1
        for k in range(r):
            v0, _ = o.random_solenoidal(seeds[q], 1.0, n / 3.0, 1, 1.0)
            ref = o.hd_run(4, 2, 1e-3, nus[q], v0)
            got = [to_host(x[k * nxh:(k + 1) * nxh]).astype(np.complex128) for x in fields]
            assert rel_l2(got, ref) < tol, (c, k)
            assert e[q] == pytest.approx(o.energy(*ref, 1), rel=max(tol, 1e-13))
            q += 1


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_tile_variants_are_bitwise_identical(prec):
    """Every tile variant (y tile width, z CTA size, two-stage z ring) gives
    the same bits, and the autotuner leaves the velocity untouched."""
    import torch
    n = 256
    g = ghost(n, precision=prec)
    V0 = [g.czeros() for _ in range(3)]
    F = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, n / 3.0, 1, 1.0, *V0)
    g.init_random_solenoidal(2000, 2.0, 3.0, 0, 1.0, *F)
    keep = [x.clone() for x in V0]
    cfg = g.hd_autotune(4, 5e-4, 1e-3, *V0, *F)
    assert cfg in (0, 1, 2, 3, 6, 7, 8, 14, 16, 22, 24, 30, 38, 46, 62, 126)
    assert all(torch.equal(a, b) for a, b in zip(V0, keep))
    ref = None
    for c in (0, 1, 2, 3, 6, 7, 8, 14, 16, 30, 38, 62, 126):
        g.set_tile_cfg(c)
        V = [x.clone() for x in keep]
        g.hd_run(2, 4, 5e-4, 1e-3, *V, *F)
        if ref is None:
            ref = V
        else:
            assert all(torch.equal(a, b) for a, b in zip(V, ref)), c


def test_wide_line_variants_at_512():
    """The FP32 y passes with 16 values per thread (bit 4), alone and with the
    other variants, give the same bits as the 8-value passes over unpruned
    and pruned substeps, and match the oracle."""
    import torch
    shape = (64, 256, 512)
    o = Oracle(*shape)
    v0, _ = o.random_solenoidal(51, 1.0, 10.0, 1, 1.0)
    f, _ = o.random_solenoidal(52, 2.0, 3.0, 0, 1.0)
    g = ghost(*shape, precision="fp32")
    F = [to_dev(x.astype(np.complex64)) for x in f]
    out = {}
    for c in (0, 14, 16, 24, 30):
        g.set_tile_cfg(c)
        V = [to_dev(x.astype(np.complex64)) for x in v0]
        g.hd_run(2, 4, 5e-4, 1e-3, *V, *F)
        out[c] = V
    for c in (14, 16, 24, 30):
        assert all(torch.equal(a, b) for a, b in zip(out[c], out[0])), c
    ref = o.hd_run(2, 4, 5e-4, 1e-3, v0, f)
    assert rel_l2([to_host(x) for x in out[30]], ref) <= 1e-5


@pytest.mark.parametrize("shape", [(1024, 16, 16), (16, 1024, 16), (16, 16, 1024)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_longest_lines(shape, prec):
    """The maximum line length (1024) along each axis, in both precisions:
    one forced RK2 step against the oracle."""
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    v0, _ = o.random_solenoidal(31, 1.0, 5.0, 1, 1.0)
    f, _ = o.random_solenoidal(32, 2.0, 3.0, 0, 1.0)
    ref = o.hd_run(1, 2, 1e-3, 1e-3, v0, f)
    cd = g.cdtype_np
    V = [to_dev(x.astype(cd)) for x in v0]
    F = [to_dev(x.astype(cd)) for x in f]
    g.hd_run(1, 2, 1e-3, 1e-3, *V, *F)
    assert rel_l2([to_host(x) for x in V], ref) <= (1e-12 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 32, 16)])
def test_transfer_spectra(prec, shape):
    """entrans (kin 1 and 0) and heltrans against the oracle on unrelated
    fields, and the zero total transfer of the nonlinear term."""
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    a = [rand_spectral(o, 70 + q) for q in range(6)]
    A = [to_dev(x.astype(g.cdtype_np)) for x in a]
    tol = 1e-12 if prec == "fp64" else 2e-6
    for kin in (1, 0):
        assert rel_l2(g.entrans(*A, kin=kin), o.entrans(*a, kin=kin)) <= tol
    assert rel_l2(g.heltrans(*A), o.heltrans(*a)) <= tol
    v = solenoidal_ic(o, seed=71)
    nl = o.prodre3(*v)
    T = g.entrans(*[to_dev(x.astype(g.cdtype_np)) for x in (*v, *nl)], kin=1)
    assert abs(T.sum()) <= (1e-11 if prec == "fp64" else 1e-5) * np.abs(T).sum()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("box", [dict(), dict(Lx=1.0, Ly=1.0, Lz=0.5, arbsize=True)])
def test_anisotropic_spectra(prec, box):
    """specpara / specperp (kin 1 and 0, hel 1) and entpara / entperp /
    heltpara / heltperp against the oracle, on a cubic and an elongated box."""
    shape = (32, 32, 16)
    o = Oracle(*shape, **box)
    g = ghost(*shape, precision=prec, **box)
    a = [rand_spectral(o, 80 + q) for q in range(6)]
    A = [to_dev(x.astype(g.cdtype_np)) for x in a]
    tol = 1e-12 if prec == "fp64" else 2e-6
    for mode, spec in ((0, g.specpara), (1, g.specperp)):
        for kin in (1, 0):
            E, H = spec(*A[:3], kin=kin, hel=1)
            Eo, Ho = o.spec_aniso(mode, *a[:3], kin=kin, hel=1)
            assert rel_l2(E, Eo) <= tol, (mode, kin)
            assert rel_l2(H, Ho) <= tol, (mode, kin)
    for mode, ent, hel in ((0, g.entpara, g.heltpara), (1, g.entperp, g.heltperp)):
        for kin in (1, 0):
            assert rel_l2(ent(*A, kin=kin), o.trans_aniso(mode, *a, kin=kin)) <= tol, (mode, kin)
        assert rel_l2(hel(*A), o.trans_aniso(mode, *a, curl=True)) <= tol, mode


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_havgcomp_and_tbouss(prec):
    """havgcomp's eleven profiles against the oracle on an elongated
    Boussinesq box, and tbouss as their z-average, maximum and minimum."""
    shape = (32, 32, 16)
    box = dict(Lx=1.0, Ly=1.0, Lz=0.5, arbsize=True)
    o = Oracle(*shape, **box)
    g = ghost(*shape, precision=prec, **box)
    v = solenoidal_ic(o, seed=13)
    s = o.random_solenoidal(14, 1.0, 4.0, 0, 1.0)[0][0]
    F = [to_dev(x.astype(g.cdtype_np)) for x in (*v, s)]
    tol = 1e-11 if prec == "fp64" else 1e-5
    prof = []
    for t in range(11):
        got = g.havgcomp(*F, 1.0, 8.0, t)
        ref = o.havgcomp(*v, s, 1.0, 8.0, t)
        assert rel_l2(got, ref) <= tol, t
        prof.append(got)
    avg, mx, mn = g.tbouss(*F, 1.0, 8.0)
    for t in range(11):
        assert np.isclose(avg[t], prof[t].mean(), rtol=1e-12, atol=0)
        assert mx[t] == prof[t].max() and mn[t] == prof[t].min()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_passive_scalar(prec):
    """The PHD solver (phd_rkstep2.f90) and the scalar diagnostics
    (variance, spectrscc, sctrans) against the oracle's restatement."""
    shape = (32, 32, 16)
    box = dict(Lx=1.0, Ly=1.0, Lz=0.5, arbsize=True)
    o = Oracle(*shape, **box)
    g = ghost(*shape, precision=prec, **box)
    v = solenoidal_ic(o, seed=23)
    th = o.random_solenoidal(24, 1.0, 4.0, 0, 1.0)[0][0]
    fs = o.random_solenoidal(25, 2.0, 3.0, 0, 0.5)[0][1]
    cd = g.cdtype_np
    V = [to_dev(x.astype(cd)) for x in v]
    TH, FS = to_dev(th.astype(cd)), to_dev(fs.astype(cd))
    g.phd_run(3, 2, 1e-3, 1e-3, 2e-3, *V, TH, fs=FS)
    rv, rth = o.phd_run(3, 2, 1e-3, 1e-3, 2e-3, v, th, fs=fs)
    tol = 1e-12 if prec == "fp64" else 1e-5
    assert rel_l2([to_host(x) for x in V], rv) <= tol
    assert rel_l2(to_host(TH), rth) <= tol
    a, b = rand_spectral(o, 26), rand_spectral(o, 27)
    A, B = to_dev(a.astype(cd)), to_dev(b.astype(cd))
    tol = 1e-12 if prec == "fp64" else 2e-6
    for kin in (1, 0):
        assert abs(g.variance(A, kin) - o.variance(a, kin)) <= tol * o.variance(a, kin)
    for shift in (0.0, 0.5):
        assert rel_l2(g.spectrscc(A, shift), o.spectrscc(a, shift)) <= tol
    assert rel_l2(g.sctrans(A, B), o.sctrans(a, b)) <= tol


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_mhd(prec):
    """GHOST's MHD operators (vector3, nonlin3, gauge3) and a forced MHD run
    (mhd_rkstep2.f90) against the oracle's restatement."""
    shape = (32, 32, 32)
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    cd = g.cdtype_np
    v = solenoidal_ic(o, seed=41)
    a = [0.3 * x for x in solenoidal_ic(o, seed=42)]
    f = o.random_solenoidal(43, 2.0, 3.0, 0, 1.0)[0]
    m = o.random_solenoidal(44, 2.0, 3.0, 0, 0.5)[0]
    r = [rand_spectral(o, 45 + q) for q in range(6)]
    R = [to_dev(x.astype(cd)) for x in r]
    tol = 1e-12 if prec == "fp64" else 2e-6
    assert rel_l2([to_host(x) for x in g.vector3(*R)], o.vector3(*r)) <= tol
    for d in (1, 2, 3):
        assert rel_l2(to_host(g.nonlin3(*R, d)), o.nonlin3(*r, d)) <= tol
        assert rel_l2(to_host(g.gauge3(*R[:3], d)), o.gauge3(*r[:3], d)) <= tol
    V = [to_dev(x.astype(cd)) for x in v]
    A = [to_dev(x.astype(cd)) for x in a]
    g.mhd_run(3, 2, 1e-3, 1e-3, 2e-3, *V, *A, f=[to_dev(x.astype(cd)) for x in f], m=[to_dev(x.astype(cd)) for x in m])
    rv, ra = o.mhd_run(3, 2, 1e-3, 1e-3, 2e-3, v, a, f=f, m=m)
    tol = 1e-11 if prec == "fp64" else 1e-5
    assert rel_l2([to_host(x) for x in V], rv) <= tol
    assert rel_l2([to_host(x) for x in A], ra) <= tol


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 16, 64)])
def test_phaseshift(prec, shape):
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    a = rand_spectral(o, 52)
    cd = 0.6 + 0.8j
    A = to_dev(a.astype(g.cdtype_np))
    g.phaseshift(A, cd)
    ref = o.phaseshift(a, cd)
    assert rel_l2(to_host(A), ref) <= (1e-15 if prec == "fp64" else 1e-7)


# ------------------------------------------- the benchmark's 512-point lines
# Shapes whose lines along one axis (or two) have 512 points run the same
# kernel instantiations as the 512^3 benchmark step: xpipe_nl_kernel<*, 512,
# ...> for nx = 512, ypipe_kernel<*, 512, ...> for ny = 512 and
# zpipe_kernel<*, 512, ...> for nz = 512.  Tile variants 30, 62 and 126 are
# the FP32 benchmark's (y passes with 16 values per thread and a second
# exchange buffer; a two-stage z ring with three CTAs per SM, or a one-stage
# z ring with four; 126 also runs the y inverse in 4-line tiles); FP64 runs
# the variants the autotuner picks at 512^3 (22, 6), the one-stage z ring
# (38) and the default.
LINE512 = [(512, 16, 16), (16, 512, 16), (16, 16, 512), (512, 512, 16)]


@pytest.mark.parametrize("shape", LINE512)
@pytest.mark.parametrize("prec,cfgs,tol", [("fp64", (0, 6, 22, 38), 1e-12), ("fp32", (0, 1, 30, 62, 126), 1e-5)])
def test_forced_rk4_with_512_point_lines(shape, prec, cfgs, tol):
    """Config 1's step (forced on 2 <= |k| <= 3, nu = 1e-3, dt = 5e-4, RK4)
    for two steps (the second zero-pruned) against the FP64 oracle; every
    tile variant gives the same bits."""
    import torch
    o = Oracle(*shape)
    kup = max(shape) / 3.0
    v0, _ = o.random_solenoidal(1000, 1.0, kup, 1, 1.0)
    f, _ = o.random_solenoidal(2000, 2.0, 3.0, 0, 1.0)
    ref = o.hd_run(2, 4, 5e-4, 1e-3, v0, f)
    g = ghost(*shape, precision=prec)
    cd = g.cdtype_np
    F = [to_dev(x.astype(cd)) for x in f]
    first = None
    for cfg in cfgs:
        g.set_tile_cfg(cfg)
        V = [to_dev(x.astype(cd)) for x in v0]
        g.hd_run(2, 4, 5e-4, 1e-3, *V, *F)
        err = rel_l2([to_host(x).astype(np.complex128) for x in V], ref)
        assert err <= tol, (cfg, err)
        if first is None:
            first = V
        else:
            assert all(torch.equal(a, b) for a, b in zip(V, first)), cfg


@pytest.mark.parametrize("shape", [(512, 16, 16), (512, 32, 32)])
def test_bouss_fp32_with_512_point_x_lines(shape):
    """The Boussinesq substep's FP32 x pass at 512-point lines (16-line tiles,
    work fields in the x-pass layout) against the FP64 oracle; tile variants
    give the same bits."""
    import torch
    o = Oracle(*shape, Lx=1, Ly=1, Lz=0.25, arbsize=True)
    v0, _ = o.random_solenoidal(57, 1.0, 40.0, 1, 1.0)
    th0 = rand_spectral(o, 58, 0.0)
    args = (4, 2.5e-4, 5e-4, 5e-4, 0.5, 8.0, 8.0)
    ref_v, ref_th = o.bouss_run(2, *args, v0, th0)
    g = ghost(*shape, Lx=1, Ly=1, Lz=0.25, arbsize=True, precision="fp32")
    first = None
    for cfg in (0, 30, 62, 126):
        g.set_tile_cfg(cfg)
        V = [to_dev(x.astype(np.complex64)) for x in v0]
        TH = to_dev(th0.astype(np.complex64))
        g.bouss_run(2, *args, *V, TH)
        got = [to_host(x).astype(np.complex128) for x in V] + [to_host(TH).astype(np.complex128)]
        assert rel_l2(got, list(ref_v) + [ref_th]) < 1e-5, cfg
        if first is None:
            first = V + [TH]
        else:
            assert all(torch.equal(a, b) for a, b in zip(V + [TH], first)), cfg


# ------------------------------------------------ rand = 2 forcing update
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_forcing_slow_matches_oracle(prec):
    """main3D.fpp:2646-2657 through ghost_forcing_slow: bit for bit with the
    oracle (no contraction), host and device arrays, output aliasing fold."""
    o = Oracle(32, precision=prec)
    g = ghost(32, precision=prec)
    a, _ = o.random_solenoidal(3, 2.0, 3.0, 0, 1.0)
    b, _ = o.random_solenoidal(4, 2.0, 3.0, 0, 1.0)
    a = [x.astype(o.cdt) for x in a]
    b = [x.astype(o.cdt) for x in b]
    for timef in (0, 2, 4):
        ref = o.forcing_slow(timef, 5, a, b)
        A = [to_dev(x) for x in a]
        out = [g.czeros() for _ in range(3)]
        g.forcing_slow(timef, 5, A, [to_dev(x) for x in b], out)
        assert all(np.array_equal(to_host(x), y) for x, y in zip(out, ref))
        g.forcing_slow(timef, 5, A, [to_dev(x) for x in b], A)  # in place over fold
        assert all(np.array_equal(to_host(x), y) for x, y in zip(A, ref))
        h = [np.zeros(o.sshape, o.cdt) for _ in range(3)]
        g.forcing_slow(timef, 5, a, b, h)  # host arrays
        assert all(np.array_equal(x, y) for x, y in zip(h, ref))


def test_rand2_forced_run_matches_oracle_loop():
    """GHOST's time loop with rand = 2 (main3D.fpp:2541-2657): every fstep
    steps the forcing is saved as fold and a new random forcing drawn with the
    continuing seed (initialfv), each step blends them; 7 forced RK2 steps at
    32^3 FP64 against the same loop on the oracle."""
    n, fstep, dt, nu = 32, 3, 1e-3, 2e-3
    o = Oracle(n)
    g = ghost(n)
    v0, _ = o.random_solenoidal(1000, 1.0, n / 3.0, 1, 1.0)
    f0, seed = o.random_solenoidal(2000, 2.0, 3.0, 0, 1.0)
    # oracle loop
    v, f, s, timef = v0, f0, seed, fstep
    fold = fnew = None
    for _ in range(7):
        if timef == fstep:
            timef = 0
            fold = [x.copy() for x in f]
            fnew, s = o.random_solenoidal(s, 2.0, 3.0, 0, 1.0)
        f = o.forcing_slow(timef, fstep, fold, fnew)
        v = o.hd_run(1, 2, dt, nu, v, f)
        timef += 1
    # library loop
    V = [to_dev(x) for x in v0]
    F = [to_dev(x) for x in f0]
    Fold = [g.czeros() for _ in range(3)]
    Fnew = [g.czeros() for _ in range(3)]
    s, timef = seed, fstep
    for _ in range(7):
        if timef == fstep:
            timef = 0
            for a, b in zip(Fold, F):
                a.copy_(b)
            s = g.init_random_solenoidal(s, 2.0, 3.0, 0, 1.0, *Fnew)
        g.forcing_slow(timef, fstep, Fold, Fnew, F)
        g.hd_run(1, 2, dt, nu, *V, *F)
        timef += 1
    assert rel_l2([to_host(x) for x in F], f) < 1e-14
    assert rel_l2([to_host(x) for x in V], v) < 1e-12


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_ensemble_one_launch_per_pass_equals_per_class_launches(prec):
    """Every pass one launch over all classes (CTAs assigned to classes by a
    tile table) against each class's own launches on its own stream: the
    same bits for four uneven classes, and each run against the oracle."""
    import torch
    from ghost_b200 import Ensemble
    sizes, nruns = [16, 32, 64, 128], [5, 3, 2, 1]
    seeds = list(range(301, 312))
    nus = [5e-4 * (1.3 ** q) for q in range(11)]
    out = {}
    for multi in (True, False):
        ens = Ensemble(sizes, nruns, precision=prec)
        ens.set_mode(multi)
        assert ens.mode() == multi
        ens.init(seeds, nus)
        ens.run(3, 2, 1e-3)
        out[multi] = [[x.clone() for x in ens.fields(c)] for c in range(len(sizes))]
        ens.close()
    for c in range(len(sizes)):
        assert all(torch.equal(a, b) for a, b in zip(out[True][c], out[False][c])), c
    tol = 1e-12 if prec == "fp64" else 1e-5
    q = 0
    for c, (n, r) in enumerate(zip(sizes, nruns)):
        o = Oracle(n)
        nxh = n // 2 + 1
        for k in range(r):
            v0, _ = o.random_solenoidal(seeds[q], 1.0, n / 3.0, 1, 1.0)
            ref = o.hd_run(3, 2, 1e-3, nus[q], v0)
            got = [to_host(x[k * nxh:(k + 1) * nxh]).astype(np.complex128) for x in out[True][c]]
            assert rel_l2(got, ref) < tol, (c, k)
            q += 1
