"""The plain 512-point FP32 x transforms with one warp per line
(fftp3d_real_to_complex / fftp3d_complex_to_real) against the oracle, and
the bounded-wait timeout path of their TMA rings."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_l2
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

def ghost(*shape, **kw):
    from ghost_b200 import Ghost
    return Ghost(*shape, **kw)


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


def test_plain_timeout_reports_and_recovers():
    """With the stall injected the warp-line transforms record
    GHOST_ERR_TIMEOUT and finish; the context then works normally."""
    from ghost_b200 import GHOST_REAL_TO_COMPLEX, GhostError
    from tests.helpers import rand_real
    shape = (512, 16, 16)
    o = Oracle(*shape)
    g = ghost(*shape, precision="fp32")
    r = rand_real(o, 7)
    plan = g.fftp3d_create_plan(shape, GHOST_REAL_TO_COMPLEX)
    out = g.czeros()
    g.set_wait_cap(1000)
    g.inject_stall(True)
    g.fftp3d_real_to_complex(plan, to_dev(r.astype(np.float32)), out)
    with pytest.raises(GhostError) as err:
        g.synchronize()
    assert err.value.code == 5
    g.inject_stall(False)
    g.set_wait_cap(0)
    g.fftp3d_real_to_complex(plan, to_dev(r.astype(np.float32)), out)
    g.synchronize()
    assert rel_l2(to_host(out), o.fftp3d_real_to_complex(r)) < 2e-6
