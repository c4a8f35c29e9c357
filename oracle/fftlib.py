"""The HD substep of GHOST on the host cores with a library FFT.

TEST AND BASELINE INFRASTRUCTURE ONLY: bench.py times it as the CPU
baseline (`--impl reference` and the `cpu_baseline` leg), and the tests
check it against the C restatement in ghost_oracle.c.  The product
(ghost_b200) never imports it.

GHOST's CPU build runs its transforms through FFTW 3.x with OpenMP threads
(fftp-3/fftp3D.fpp:91-107: dfftw_plan_many_dft_r2c over (x, y) per z-plane,
a transpose, dfftw_plan_many_dft along z).  FFTW is not on this machine; the
nearest threaded FFT library present is scipy's pocketfft, so this module
restates the same steps with scipy.fft (workers = all host threads) and
numpy elementwise work split over the same threads:
  fftp3d_real_to_complex  (fftp3D.fpp:204-315): rfft2 over (x, y) per
                           z-plane, transpose to a(nz, ny, nx/2+1), fft
                           along z, unnormalised;
  fftp3d_complex_to_real  (fftp3D.fpp:318-431): the same in reverse;
  prodre3, nonlhd3, laplak3 and the truncated update of hd_rkstep2
                           (pseudospec3D_hd.f90:316-509,
                           include/hd_rkstep2.f90:3-32).
Arrays use the C-order shapes of oracle.Oracle: spectral (nx/2+1, ny, nz),
real (nz, ny, nx).
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft


class FFTLibHD:
    def __init__(self, oracle, threads: int | None = None):
        """oracle: an oracle.Oracle of the same grid, for GHOST's wavenumber
        tables (kx, ky, kz, kk2, kn2, kmax, tiny)."""
        self.o = oracle
        self.nx, self.ny, self.nz = oracle.nx, oracle.ny, oracle.nz
        self.nxh = self.nx // 2 + 1
        self.rdt, self.cdt = oracle.rdt, oracle.cdt
        self.threads = threads or os.cpu_count() or 1
        self.pool = ThreadPoolExecutor(self.threads)
        kx, ky, kz, kn2, kk2 = oracle.tables()
        self.kx = kx[:self.nxh].astype(self.rdt)[:, None, None]
        self.ky = ky.astype(self.rdt)[None, :, None]
        self.kz = kz.astype(self.rdt)[None, None, :]
        self.kk2 = kk2.astype(self.rdt)
        self.keep = (kn2 <= oracle.kmax) & (kn2 >= oracle.tiny)
        nn = self.rdt(self.nx) * self.rdt(self.ny) * self.rdt(self.nz)
        self.tmp = self.rdt(1) / (nn * nn)

    # elementwise work over slabs of the slowest axis, one per thread
    def par(self, fn, *arrays):
        n = arrays[0].shape[0]
        q = max(1, (n + self.threads - 1) // self.threads)
        futs = [self.pool.submit(fn, slice(s, min(n, s + q))) for s in range(0, n, q)]
        for f in futs:
            f.result()

    def r2c(self, r):
        """fftp3d_real_to_complex of r (nz, ny, nx) -> a (nx/2+1, ny, nz)."""
        c = sfft.rfft2(r, axes=(1, 2), workers=self.threads)  # (nz, ny, nxh), per z-plane
        out = np.empty((self.nxh, self.ny, self.nz), self.cdt)
        self.par(lambda s: out.__setitem__(s, c[:, :, s].transpose(2, 1, 0)), out)
        return sfft.fft(out, axis=2, workers=self.threads, overwrite_x=True)

    def c2r(self, a):
        """fftp3d_complex_to_real of a (nx/2+1, ny, nz) -> r (nz, ny, nx)."""
        t = sfft.ifft(a, axis=2, norm="forward", workers=self.threads)
        c = np.empty((self.nz, self.ny, self.nxh), self.cdt)
        self.par(lambda s: c.__setitem__(s, t[:, :, s].transpose(2, 1, 0)), c)
        # pocketfft's c2r along x reads only the real parts of kx = 0 and
        # nx/2 after the y transform, as GHOST's c2r of Hermitian lines does
        return sfft.irfft2(c, s=(self.ny, self.nx), axes=(1, 2), norm="forward", workers=self.threads,
                           overwrite_x=True)

    def curl(self, a, b, c):
        """rotor3 for the three directions: (dy c - dz b, dz a - dx c, dx b - dy a)."""
        kx, ky, kz = self.kx, self.ky, self.kz
        w = [np.empty_like(a) for _ in range(3)]

        def f(s):
            A, B, Cc = a[s], b[s], c[s]
            KX = kx[s]
            w[0][s] = 1j * (ky * Cc - kz * B)
            w[1][s] = 1j * (kz * A - KX * Cc)
            w[2][s] = 1j * (KX * B - ky * A)
        self.par(f, a)
        return w

    def prodre3(self, a, b, c):
        """[curl(v) x v] in Fourier space (pseudospec3D_hd.f90:316-396)."""
        w1, w2, w3 = (self.c2r(x) for x in self.curl(a, b, c))
        r4, r5, r6 = self.c2r(a), self.c2r(b), self.c2r(c)
        tmp = self.tmp
        p1, p2, p3 = np.empty_like(r4), np.empty_like(r4), np.empty_like(r4)

        def f(s):
            p1[s] = (w2[s] * r6[s] - r5[s] * w3[s]) * tmp
            p2[s] = (w3[s] * r4[s] - r6[s] * w1[s]) * tmp
            p3[s] = (w1[s] * r5[s] - r4[s] * w2[s]) * tmp
        self.par(f, r4)
        return self.r2c(p1), self.r2c(p2), self.r2c(p3)

    def hd_rkstep2(self, o, dt, nu, v, C, f):
        """One substep: nonlhd3 x3 of prodre3, laplak3, truncated update."""
        n1, n2, n3 = self.prodre3(*v)
        kx, ky, kz, kk2, keep = self.kx, self.ky, self.kz, self.kk2, self.keep
        rdt = self.rdt
        dt, nu, rmp = rdt(dt), rdt(nu), rdt(1) / rdt(o)
        out = [np.empty_like(x) for x in v]

        def g(s):
            KX = kx[s]
            k2 = kk2[s]
            safe = np.where(k2 > 0, k2, rdt(1))
            kdot = (KX * n1[s] + ky * n2[s] + kz * n3[s]) / safe
            # nonlhd3: -a_dir + k_dir (k.a)/k^2, the k_dir = 0 plane -a_dir
            nl = (-n1[s] + KX * kdot, -n2[s] + ky * kdot, -n3[s] + kz * kdot)
            for q in range(3):
                upd = C[q][s] + rmp * (dt * ((nu * (-k2 * v[q][s]) + nl[q]) + f[q][s]))
                out[q][s] = np.where(keep[s], upd, 0)
        self.par(g, v[0])
        return out

    def hd_run(self, nsteps, ord, dt, nu, v, f):
        v = [np.ascontiguousarray(x, self.cdt) for x in v]
        f = [np.ascontiguousarray(x, self.cdt) for x in f]
        for _ in range(nsteps):
            C = [x.copy() for x in v]
            for o in range(ord, 0, -1):
                v = self.hd_rkstep2(o, dt, nu, v, C, f)
        return v

    def close(self):
        self.pool.shutdown()
