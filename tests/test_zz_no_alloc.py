"""ghost_spectrumc_noalloc: the shell spectra for callers that cannot let the
library allocate device memory (runs whose fields already fill HBM, or that
cannot take an allocation's device-wide synchronisation inside the time
loop).  Called through the C ABI and checked against ghost_spectrumc on two
calls in a row, plus the rejections the header promises.  Collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spectra_noalloc(g, lib, v, kin, hel):
    nb = g.nmax // 2 + 1
    Ek, Hk = np.zeros(nb), np.zeros(nb)
    pd = ctypes.POINTER(ctypes.c_double)
    s = lib.ghost_spectrumc_noalloc(g.h, *[ctypes.c_void_p(x.data_ptr()) for x in v], kin, hel,
                                    Ek.ctypes.data_as(pd), Hk.ctypes.data_as(pd))
    return s, Ek, Hk


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_noalloc_spectrum_matches_allocating_entry_point(prec):
    import torch

    from ghost_b200 import Ghost, _lib
    lib = _lib.load()
    g = Ghost(64, precision=prec)
    v = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, 64 / 3.0, 1, 1.0, *v)
    Ek0, Hk0 = g.spectrumc(*v, 1, 1)   # existing entry point (allocates its partials on first use)
    Ew0, _ = g.spectrumc(*v, 0, 0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):                   # two calls in a row share the static scratch
        s, Ek, Hk = _spectra_noalloc(g, lib, v, 1, 1)
        assert s == 0, lib.ghost_last_error_string()
        assert np.allclose(Ek, Ek0, rtol=1e-12, atol=0)
        assert np.allclose(Hk, Hk0, rtol=1e-9, atol=1e-18)
        s, Ew, _ = _spectra_noalloc(g, lib, v, 0, 0)
        assert s == 0
        assert np.allclose(Ew, Ew0, rtol=1e-12, atol=0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_spectrum_on_a_batched_context_sums_every_run():
    """A batch of three 32^3 runs: both entry points bin the modes of every
    run, so the spectra agree with each other and with the sum of the three
    runs' own spectra."""
    from ghost_b200 import Ghost, _lib
    lib = _lib.load()
    seeds = [21, 22, 23]
    g = Ghost(32, precision="fp64", nruns=3)
    v = [g.czeros() for _ in range(3)]
    g.batch_init_random_solenoidal(seeds, 1.0, 32 / 3.0, 1, 1.0, *v)
    Ek0, Hk0 = g.spectrumc(*v, 1, 1)
    for _ in range(2):
        s, Ek, Hk = _spectra_noalloc(g, lib, v, 1, 1)
        assert s == 0, lib.ghost_last_error_string()
        assert np.allclose(Ek, Ek0, rtol=1e-12, atol=0)
        assert np.allclose(Hk, Hk0, rtol=1e-9, atol=1e-18)
    one = Ghost(32, precision="fp64")
    nxh = 17
    total = np.zeros_like(Ek0)
    for r in range(3):
        e, _ = one.spectrumc(*[x[r * nxh:(r + 1) * nxh].contiguous() for x in v], 1, 0)
        total += e
    assert np.allclose(Ek, total, rtol=1e-12, atol=0)


def test_noalloc_spectrum_rejects_what_it_cannot_do():
    from ghost_b200 import Ghost, _lib
    lib = _lib.load()
    # a 16 x 16 x 1024 box with Lz = 1/4 has nmax = 4096: 2049 shells > 1008
    g = Ghost(16, 16, 1024, Lx=1, Ly=1, Lz=0.25, arbsize=True, precision="fp32")
    v = [g.czeros() for _ in range(3)]
    s, _, _ = _spectra_noalloc(g, lib, v, 1, 0)
    assert s == 2 and b"shells" in lib.ghost_last_error_string()
    # host arrays would need staging buffers
    h = Ghost(32)
    arrs = [np.zeros(h.sshape, np.complex128) for _ in range(3)]
    Ek = np.zeros(h.nmax // 2 + 1)
    pd = ctypes.POINTER(ctypes.c_double)
    s = lib.ghost_spectrumc_noalloc(h.h, *[ctypes.c_void_p(a.ctypes.data) for a in arrs], 1, 0,
                                    Ek.ctypes.data_as(pd), None)
    assert s == 1 and b"device arrays" in lib.ghost_last_error_string()
