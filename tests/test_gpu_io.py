"""GHOST's binary field files (mpiio/binary_io.f90) through the library:
the output step (main3D.fpp:2678-2709) and the restart (main3D.fpp:2155-2161)
against the oracle's transforms, raw-file layout read back with numpy, byte
swapping, host and device arrays, and the error paths."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_l2
from tests.helpers import rand_real, to_dev, to_host

pytestmark = pytest.mark.gpu


def ghost(*shape, **kw):
    from ghost_b200 import Ghost
    return Ghost(*shape, **kw)


@pytest.mark.parametrize("prec,shape", [("fp64", (64, 32, 16)), ("fp32", (64, 32, 16)), ("fp32", (512, 16, 32))])
def test_output_step(tmp_path, prec, shape):
    """The file holds the real field of v/(nx ny nz), x fastest, GP values."""
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    v, _ = o.random_solenoidal(61, 1.0, 5.0, 1, 1.0)
    V = to_dev(v[0].astype(g.cdtype_np))
    keep = V.clone()
    path = str(tmp_path / "vx.0001.out")
    g.io_output(V, path)
    got = np.fromfile(path, dtype=g.rdtype_np).reshape(shape[::-1])
    ref = o.fftp3d_complex_to_real(v[0] / float(np.prod(shape)))
    assert rel_l2(got, ref) <= (1e-13 if prec == "fp64" else 2e-6)
    assert bool((V == keep).all())


@pytest.mark.parametrize("prec,shape", [("fp64", (32, 64, 16)), ("fp32", (512, 32, 16))])
def test_restart(tmp_path, prec, shape):
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    r = rand_real(o, 62).astype(g.rdtype_np)
    path = str(tmp_path / "vy.0003.out")
    r.tofile(path)
    S = g.io_restart(path)
    ref = o.fftp3d_real_to_complex(r.astype(np.float64))
    assert rel_l2(to_host(S), ref) <= (1e-13 if prec == "fp64" else 2e-6)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_output_then_restart_round_trip(tmp_path, prec):
    shape = (512, 16, 32) if prec == "fp32" else (64, 64, 32)
    o = Oracle(*shape)
    g = ghost(*shape, precision=prec)
    v, _ = o.random_solenoidal(63, 1.0, 5.0, 1, 1.0)
    V = to_dev(v[1].astype(g.cdtype_np))
    path = str(tmp_path / "vz.0002.out")
    g.io_output(V, path)
    back = g.io_restart(path)
    assert rel_l2(to_host(back), to_host(V)) <= (1e-14 if prec == "fp64" else 1e-6)


def test_swap_and_host_arrays(tmp_path):
    shape = (32, 32, 32)
    o = Oracle(*shape)
    g = ghost(*shape, precision="fp64")
    r = rand_real(o, 64)
    p1 = str(tmp_path / "a.out")
    p2 = str(tmp_path / "b.out")
    g.io_write(to_dev(r), p1)
    g.io_write(r, p2, swap=True)  # a host array, byte-swapped
    a = np.fromfile(p1, dtype=np.float64).reshape(r.shape)
    b = np.fromfile(p2, dtype=np.float64).byteswap().reshape(r.shape)
    assert np.array_equal(a, r) and np.array_equal(b, r)
    back = g.io_read(p2, swap=True)
    assert np.array_equal(to_host(back), r)
    host = np.zeros_like(r)
    g.io_read(p1, out=host)
    assert np.array_equal(host, r)
    # host spectral arrays for the output step and the restart
    v, _ = o.random_solenoidal(65, 1.0, 5.0, 1, 1.0)
    g.io_output(v[2], p1)
    g.io_output(to_dev(v[2]), p2)
    assert open(p1, "rb").read() == open(p2, "rb").read()
    hs = np.zeros(o.sshape, np.complex128)
    g.io_restart(p1, out=hs)
    assert np.array_equal(hs, to_host(g.io_restart(p1)))


def test_errors(tmp_path):
    from ghost_b200 import GhostError
    g = ghost(32, 32, 32, precision="fp32")
    bad = tmp_path / "short.out"
    np.zeros(100, np.float32).tofile(bad)
    with pytest.raises(GhostError) as e:
        g.io_read(str(bad))
    assert e.value.code == 2
    with pytest.raises(GhostError) as e:
        g.io_restart(str(tmp_path / "missing.out"))
    assert e.value.code == 9
    with pytest.raises(GhostError) as e:
        g.io_output(g.czeros(), str(tmp_path / "no_such_dir" / "x.out"))
    assert e.value.code == 9
