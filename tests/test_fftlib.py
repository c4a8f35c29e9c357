"""The library-FFT CPU leg that bench.py times as the CPU baseline
(oracle/fftlib.py: GHOST's steps with scipy's pocketfft in place of FFTW)
computes what the C oracle computes: the transforms, prodre3 and whole
forced RK4 steps, FP64 within 1e-12 and FP32 within 1e-5."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_l2


@pytest.mark.parametrize("shape", [(16, 8, 32), (32, 32, 32), (64, 16, 8)])
def test_transforms_and_prodre3_match_the_oracle(shape):
    from oracle.fftlib import FFTLibHD
    o = Oracle(*shape)
    lib = FFTLibHD(o, threads=2)
    rng = np.random.default_rng(5)
    r = rng.standard_normal(o.rshape)
    assert rel_l2(lib.r2c(r), o.fftp3d_real_to_complex(r)) < 1e-14
    c = rng.standard_normal(o.sshape) + 1j * rng.standard_normal(o.sshape)  # not Hermitian
    assert rel_l2(lib.c2r(c), o.fftp3d_complex_to_real(c)) < 1e-14
    v, _ = o.random_solenoidal(1000, 1.0, max(shape) / 3.0, 1, 1.0)
    assert rel_l2(list(lib.prodre3(*v)), list(o.prodre3(*v))) < 1e-13
    lib.close()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_forced_rk4_steps_match_the_oracle(prec, tol):
    from oracle.fftlib import FFTLibHD
    o = Oracle(32, 16, 64, precision=prec)
    ref64 = Oracle(32, 16, 64)
    lib = FFTLibHD(o, threads=2)
    v, _ = ref64.random_solenoidal(1000, 1.0, 32 / 3.0, 1, 1.0)
    f, _ = ref64.random_solenoidal(2000, 2.0, 3.0, 0, 1.0)
    ref = ref64.hd_run(2, 4, 5e-4, 1e-3, v, f)
    got = lib.hd_run(2, 4, 5e-4, 1e-3, v, f)
    assert rel_l2([x.astype(np.complex128) for x in got], ref) < tol
    # the truncation: nothing outside tiny <= kn2 <= kmax
    assert all(np.all(x[~lib.keep] == 0) for x in got)
    lib.close()
