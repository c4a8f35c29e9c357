"""The fused x pass with one warp per x line (tile variant bit 4; FP32,
512-point x lines): the same bits as the cross-warp x pass, parity with the
oracle, unpruned and pruned substeps, an ensemble, and the bounded-wait
timeout path of its TMA ring."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_l2
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

XW = 16


def ghost(*shape, **kw):
    from ghost_b200 import Ghost
    return Ghost(*shape, **kw)


@pytest.mark.parametrize("shape", [(512, 32, 32), (512, 16, 64), (512, 128, 16)])
def test_same_bits_as_cross_warp_pass(shape):
    import torch
    g = ghost(*shape, precision="fp32")
    V0 = [g.czeros() for _ in range(3)]
    F = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, min(shape) / 3.0, 1, 1.0, *V0)
    g.init_random_solenoidal(2000, 2.0, 3.0, 0, 1.0, *F)
    out = {}
    for cfg in (0, XW, 14, 14 | XW):
        g.set_tile_cfg(cfg)
        V = [x.clone() for x in V0]
        g.hd_run(2, 4, 5e-4, 1e-3, *V, *F)  # the first substep unpruned, the rest pruned
        out[cfg] = V
    for cfg in (XW, 14, 14 | XW):
        assert all(torch.equal(a, b) for a, b in zip(out[cfg], out[0])), cfg


def test_oracle_parity():
    shape = (512, 32, 32)
    o = Oracle(*shape)
    g = ghost(*shape, precision="fp32")
    g.set_tile_cfg(XW)
    v0, _ = o.random_solenoidal(41, 1.0, 8.0, 1, 1.0)
    f, _ = o.random_solenoidal(42, 2.0, 3.0, 0, 1.0)
    ref = o.hd_run(2, 2, 1e-3, 1e-3, v0, f)
    V = [to_dev(x.astype(np.complex64)) for x in v0]
    F = [to_dev(x.astype(np.complex64)) for x in f]
    g.hd_run(2, 2, 1e-3, 1e-3, *V, *F)
    assert rel_l2([to_host(x) for x in V], ref) <= 1e-5


def test_ensemble_runs():
    """Four runs batched in one context: each run matches a solo run."""
    import torch
    from ghost_b200 import Ghost
    shape = (512, 16, 16)
    ge = Ghost(*shape, precision="fp32", nruns=4)
    ge.set_tile_cfg(XW)
    g1 = ghost(*shape, precision="fp32")
    g1.set_tile_cfg(0)
    runs = []
    for r in range(4):
        v = [g1.czeros() for _ in range(3)]
        g1.init_random_solenoidal(500 + r, 1.0, 5.0, 1, 1.0, *v)
        runs.append(v)
    Ve = [torch.cat([runs[r][a] for r in range(4)]) for a in range(3)]
    ge.hd_run(2, 2, 1e-3, 1e-3, *Ve)
    for r in range(4):
        v = [x.clone() for x in runs[r]]
        g1.hd_run(2, 2, 1e-3, 1e-3, *v)
        h = v[0].shape[0]  # runs are stacked along kx
        for a in range(3):
            assert torch.equal(Ve[a][r * h:(r + 1) * h], v[a]), (r, a)


def test_timeout_reports_and_recovers():
    from ghost_b200 import GhostError
    shape = (512, 16, 16)
    o = Oracle(*shape)
    g = ghost(*shape, precision="fp32")
    g.set_tile_cfg(XW)
    v0, _ = o.random_solenoidal(43, 1.0, 5.0, 1, 1.0)
    V = [to_dev(x.astype(np.complex64)) for x in v0]
    g.set_wait_cap(1000)
    g.inject_stall(True)
    g.hd_run(1, 2, 1e-3, 2e-3, *V)
    with pytest.raises(GhostError) as err:
        g.synchronize()
    assert err.value.code == 5
    g.inject_stall(False)
    g.set_wait_cap(0)
    V = [to_dev(x.astype(np.complex64)) for x in v0]
    g.hd_run(1, 2, 1e-3, 2e-3, *V)
    g.synchronize()
    ref = o.hd_run(1, 2, 1e-3, 2e-3, v0)
    assert rel_l2([to_host(x) for x in V], ref) < 1e-5


@pytest.mark.parametrize("shape", [(512, 16, 32), (512, 32, 16)])
def test_plain_r2c_warp_lines(shape):
    """fftp3d_real_to_complex at nx = 512 (FP32) runs the warp-line x pass."""
    from ghost_b200 import GHOST_REAL_TO_COMPLEX
    from tests.helpers import rand_real
    o = Oracle(*shape)
    g = ghost(*shape, precision="fp32")
    r = rand_real(o, 5)
    ref = o.fftp3d_real_to_complex(r)
    plan = g.fftp3d_create_plan(shape, GHOST_REAL_TO_COMPLEX)
    out = g.czeros()
    g.fftp3d_real_to_complex(plan, to_dev(r.astype(np.float32)), out)
    assert rel_l2(to_host(out), ref) < 2e-6


@pytest.mark.parametrize("shape", [(512, 16, 32), (512, 32, 16)])
def test_plain_c2r_warp_lines(shape):
    """fftp3d_complex_to_real at nx = 512 (FP32), a non-Hermitian input
    (only the real parts of the kx = 0 and Nyquist values count)."""
    from ghost_b200 import GHOST_COMPLEX_TO_REAL
    from tests.helpers import rand_spectral
    o = Oracle(*shape)
    g = ghost(*shape, precision="fp32")
    c = rand_spectral(o, 6)
    ref = o.fftp3d_complex_to_real(c)
    plan = g.fftp3d_create_plan(shape, GHOST_COMPLEX_TO_REAL)
    cin = to_dev(c.astype(np.complex64))
    keep = cin.clone()
    out = g.rzeros()
    g.fftp3d_complex_to_real(plan, cin, out)
    assert rel_l2(to_host(out), ref) < 2e-6
    assert bool((cin == keep).all())
