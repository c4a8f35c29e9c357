"""The oracle's transforms against the DFT definition (what FFTW computes for
GHOST's fftp-3 path): direct O(N^2) sums at small sizes and scipy's
pocketfft at larger ones.  Layout: GHOST's transposed spectrum (nz,ny,nx/2+1)."""
import numpy as np
import pytest
import scipy.fft

from oracle.oracle import Oracle


def dft_matrix(n, sign):
    k = np.arange(n)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / n)


def direct_r2c(r):
    nz, ny, nx = r.shape
    Fx, Fy, Fz = dft_matrix(nx, -1), dft_matrix(ny, -1), dft_matrix(nz, -1)
    X = np.einsum("zyx,ax,by,cz->abc", r, Fx, Fy, Fz)
    return X[: nx // 2 + 1]  # (kx, ky, kz) == GHOST (nx/2+1, ny, nz) C-order


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 8, 32), (8, 16, 16)])
def test_r2c_matches_direct_dft(shape):
    nx, ny, nz = shape
    o = Oracle(nx, ny, nz)
    r = np.random.default_rng(1).standard_normal(o.rshape)
    out = o.fftp3d_real_to_complex(r)
    ref = direct_r2c(r)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("n", [32, 64])
def test_r2c_matches_pocketfft(n):
    o = Oracle(n)
    r = np.random.default_rng(2).standard_normal(o.rshape)
    ref = scipy.fft.rfftn(r, axes=(0, 1, 2)).transpose(2, 1, 0)
    out = o.fftp3d_real_to_complex(r)
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 32, 8), (32, 32, 32)])
def test_c2r_is_unnormalised_inverse(shape):
    o = Oracle(*shape)
    r = np.random.default_rng(3).standard_normal(o.rshape)
    back = o.fftp3d_complex_to_real(o.fftp3d_real_to_complex(r))
    assert np.abs(back / r.size - r).max() < 1e-13


def test_c2r_ignores_imaginary_parts_of_kx0_and_nyquist():
    """A complex-to-real transform of Hermitian data reads only the real parts
    of the kx=0 and kx=nx/2 coefficients (after the y,z transforms); pocketfft's
    irfftn does the same, so it is the definition used here."""
    o = Oracle(16, 8, 8)
    rng = np.random.default_rng(4)
    c = (rng.standard_normal(o.sshape) + 1j * rng.standard_normal(o.sshape))
    ref = scipy.fft.irfftn(c.transpose(2, 1, 0), s=(o.nz, o.ny, o.nx), axes=(0, 1, 2)) * (o.nx * o.ny * o.nz)
    out = o.fftp3d_complex_to_real(c)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


def test_fp32_oracle_close_to_fp64():
    o64, o32 = Oracle(32), Oracle(32, precision="fp32")
    r = np.random.default_rng(5).standard_normal(o64.rshape)
    a = o64.fftp3d_real_to_complex(r)
    b = o32.fftp3d_real_to_complex(r.astype(np.float32))
    assert np.abs(a - b).max() / np.abs(a).max() < 1e-5
