"""ctypes front end of the CPU restatement in ghost_oracle.c.

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py use it as the checker.
The product (ghost_b200) never imports it.

Arrays follow GHOST's Fortran layouts expressed as C-order numpy shapes:
  spectral a(nz,ny,nx/2+1) column-major  ->  numpy shape (nx//2+1, ny, nz)
  real     r(nx,ny,nz)     column-major  ->  numpy shape (nz, ny, nx)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[str, ctypes.CDLL] = {}


def build() -> None:
    """Compile liboracle_f64.so / liboracle_f32.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(precision: str) -> ctypes.CDLL:
    name = {"fp64": "liboracle_f64.so", "fp32": "liboracle_f32.so"}[precision]
    if precision not in _LIBS:
        path = os.path.join(_HERE, name)
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        _declare(lib, precision)
        _LIBS[precision] = lib
    return _LIBS[precision]


P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double


def _declare(lib: ctypes.CDLL, precision: str) -> None:
    sig = {
        "o_ctx_create": (P, [I, I, I, D, D, D, I, I]),
        "o_ctx_destroy": (None, [P]),
        "o_ctx_info": (None, [P, P]),
        "o_ctx_tables": (None, [P, P, P, P, P, P]),
        "o_nthreads": (I, []),
        "o_set_threads": (None, [I]),
        "o_fftp3d_real_to_complex": (None, [P, P, P]),
        "o_fftp3d_complex_to_real": (None, [P, P, P]),
        "o_derivk3": (None, [P, P, P, I]),
        "o_laplak3": (None, [P, P, P]),
        "o_rotor3": (None, [P, P, P, P, I]),
        "o_prodre3": (None, [P, P, P, P, P, P, P]),
        "o_nonlhd3": (None, [P, P, P, P, P, I]),
        "o_energy": (D, [P, P, P, P, I]),
        "o_helicity": (D, [P, P, P, P]),
        "o_cross": (D, [P, P, P, P, P, P, P, I]),
        "o_divergence": (D, [P, P, P, P]),
        "o_maxabs": (D, [P, P, P, P, I]),
        "o_spectrumc": (None, [P, P, P, P, I, I, P, P]),
        "o_entrans": (None, [P, P, P, P, P, P, P, I, P]),
        "o_heltrans": (None, [P, P, P, P, P, P, P, P]),
        "o_spec_aniso": (None, [P, I, P, P, P, I, I, P, P]),
        "o_havgcomp": (None, [P, P, P, P, P, D, D, I, P]),
        "o_phd_run": (None, [P, I, I, D, D, D] + [P] * 8),
        "o_vector3": (None, [P] * 10),
        "o_phaseshift": (None, [P, P, D, D]),
        "o_forcing_slow": (None, [P, I, I, P, P, P]),
        "o_nonlin3": (None, [P] * 8 + [I]),
        "o_gauge3": (None, [P] * 5 + [I]),
        "o_mhd_run": (None, [P, I, I, D, D, D] + [P] * 12),
        "o_variance": (D, [P, P, I]),
        "o_spectrscc": (None, [P, P, D, P]),
        "o_sctrans": (None, [P, P, P, P]),
        "o_trans_aniso": (None, [P, I, P, P, P, P, P, P, I, I, P]),
        "o_randu": (ctypes.c_double if precision == "fp64" else ctypes.c_float, [P]),
        "o_random_vpot": (ctypes.c_int32, [P, ctypes.c_int32, D, D, I, P, P, P]),
        "o_random_solenoidal": (ctypes.c_int32, [P, ctypes.c_int32, D, D, I, D, P, P, P]),
        "o_normalize": (None, [P, P, P, P, D, I]),
        "o_abc": (None, [P, D, D, D, D, D, P, P, P]),
        "o_hd_rkstep1": (None, [P, P, P, P, P, P, P]),
        "o_hd_rkstep2": (None, [P, I, D, D, P, P, P, P, P, P, P, P, P]),
        "o_hd_run": (None, [P, I, I, D, D, P, P, P, P, P, P]),
        "o_advect3": (None, [P, P, P, P, P, P]),
        "o_bouss_rkstep2": (None, [P, I, D, D, D, D, D, D] + [P] * 12),
        "o_bouss_run": (None, [P, I, I, D, D, D, D, D, D] + [P] * 8),
        "o_sharp": (None, [P, P, P, D]),
        "o_evedqnm": (None, [P, D, P, D, D, P, P, P]),
        "o_edqnm_rkstep2": (None, [P, I, D, D, P, P, P, I] + [P] * 9),
        "o_edqnm_run": (None, [P, I, I, D, D, D, D, I] + [P] * 6),
        "o_evedqnm_h": (None, [P, D, P, P, D, D, I, P, P, P, P, P, P]),
        "o_edqnm_run_h": (None, [P, I, I, D, D, D, D, I, I] + [P] * 6),
        "o_vcorrect": (None, [P, P, P, P, P, P, P, D]),
        "o_les_truncate": (None, [P, P, P, P, I]),
        "o_ctx_set_kmax": (None, [P, D]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class Oracle:
    """GHOST's grid/kes/ali/boxsize state plus the HD routines, on the CPU."""

    def __init__(self, nx: int, ny: int | None = None, nz: int | None = None,
                 Lx: float = 1.0, Ly: float = 1.0, Lz: float = 1.0,
                 arbsize: bool = False, edqnm: bool = False, precision: str = "fp64"):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nxh = nx // 2 + 1
        self.precision = precision
        self.rdt = np.float64 if precision == "fp64" else np.float32
        self.cdt = np.complex128 if precision == "fp64" else np.complex64
        self.lib = _lib(precision)
        self.h = self.lib.o_ctx_create(nx, ny, nz, Lx, Ly, Lz, int(arbsize), int(edqnm))
        if not self.h:
            raise ValueError(f"oracle: unsupported grid {nx}x{ny}x{nz}")
        info = np.zeros(9)
        self.lib.o_ctx_info(self.h, info.ctypes.data)
        self.kmax, self.tiny, self.Dkk = float(info[0]), float(info[1]), float(info[2])
        self.nmax, self.anis, self.nmaxperp = int(info[3]), int(info[4]), int(info[5])
        self.Dkx, self.Dky, self.Dkz = float(info[6]), float(info[7]), float(info[8])

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.o_ctx_destroy(h)
            self.h = None

    # shapes -----------------------------------------------------------
    @property
    def sshape(self):
        return (self.nxh, self.ny, self.nz)

    @property
    def rshape(self):
        return (self.nz, self.ny, self.nx)

    def czeros(self):
        return np.zeros(self.sshape, dtype=self.cdt)

    def rzeros(self):
        return np.zeros(self.rshape, dtype=self.rdt)

    def _c(self, a):
        return np.ascontiguousarray(a, dtype=self.cdt)

    def _r(self, a):
        return np.ascontiguousarray(a, dtype=self.rdt)

    def tables(self):
        kx = np.zeros(self.nx, self.rdt)
        ky = np.zeros(self.ny, self.rdt)
        kz = np.zeros(self.nz, self.rdt)
        kn2 = np.zeros(self.sshape, self.rdt)
        kk2 = np.zeros(self.sshape, self.rdt)
        self.lib.o_ctx_tables(self.h, _ptr(kx), _ptr(ky), _ptr(kz), _ptr(kn2), _ptr(kk2))
        return kx, ky, kz, kn2, kk2

    # fftp ---------------------------------------------------------------
    def fftp3d_real_to_complex(self, r):
        r = self._r(r)
        out = self.czeros()
        self.lib.o_fftp3d_real_to_complex(self.h, _ptr(r), _ptr(out))
        return out

    def fftp3d_complex_to_real(self, c):
        c = self._c(c)
        out = self.rzeros()
        self.lib.o_fftp3d_complex_to_real(self.h, _ptr(c), _ptr(out))
        return out

    # pseudospec3D_hd ----------------------------------------------------
    def derivk3(self, a, dir):
        a = self._c(a)
        b = self.czeros()
        self.lib.o_derivk3(self.h, _ptr(a), _ptr(b), dir)
        return b

    def laplak3(self, a):
        a = self._c(a)
        b = self.czeros()
        self.lib.o_laplak3(self.h, _ptr(a), _ptr(b))
        return b

    def rotor3(self, a, b, dir):
        a, b = self._c(a), self._c(b)
        c = self.czeros()
        self.lib.o_rotor3(self.h, _ptr(a), _ptr(b), _ptr(c), dir)
        return c

    def prodre3(self, a, b, c):
        a, b, c = self._c(a), self._c(b), self._c(c)
        d, e, f = self.czeros(), self.czeros(), self.czeros()
        self.lib.o_prodre3(self.h, _ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(e), _ptr(f))
        return d, e, f

    def nonlhd3(self, a, b, c, dir):
        a, b, c = self._c(a), self._c(b), self._c(c)
        g = self.czeros()
        self.lib.o_nonlhd3(self.h, _ptr(a), _ptr(b), _ptr(c), _ptr(g), dir)
        return g

    def energy(self, a, b, c, kin):
        a, b, c = self._c(a), self._c(b), self._c(c)
        return self.lib.o_energy(self.h, _ptr(a), _ptr(b), _ptr(c), kin)

    def helicity(self, a, b, c):
        a, b, c = self._c(a), self._c(b), self._c(c)
        return self.lib.o_helicity(self.h, _ptr(a), _ptr(b), _ptr(c))

    def cross(self, a, b, c, d, e, f, kin):
        arrs = [self._c(x) for x in (a, b, c, d, e, f)]
        return self.lib.o_cross(self.h, *[_ptr(x) for x in arrs], kin)

    def divergence(self, a, b, c):
        a, b, c = self._c(a), self._c(b), self._c(c)
        return self.lib.o_divergence(self.h, _ptr(a), _ptr(b), _ptr(c))

    def maxabs(self, a, b, c, kin):
        a, b, c = self._c(a), self._c(b), self._c(c)
        return self.lib.o_maxabs(self.h, _ptr(a), _ptr(b), _ptr(c), kin)

    def spectrumc(self, a, b, c, kin=1, hel=0):
        a, b, c = self._c(a), self._c(b), self._c(c)
        nb = self.nmax // 2 + 1
        Ek = np.zeros(nb)
        Hk = np.zeros(nb)
        self.lib.o_spectrumc(self.h, _ptr(a), _ptr(b), _ptr(c), kin, hel, _ptr(Ek), _ptr(Hk))
        return Ek, Hk

    def entrans(self, a, b, c, d, e, f, kin=1):
        """entrans: Ektot (shell sums of the transfer, pseudospec3D_hd.f90:1629-1820)."""
        arrs = [self._c(x) for x in (a, b, c, d, e, f)]
        Ek = np.zeros(self.nmax // 2 + 1)
        self.lib.o_entrans(self.h, *[_ptr(x) for x in arrs], kin, _ptr(Ek))
        return Ek

    def heltrans(self, a, b, c, d, e, f):
        """heltrans: Hktot, the same with curl(a,b,c) (:1823-1949)."""
        arrs = [self._c(x) for x in (a, b, c, d, e, f)]
        Hk = np.zeros(self.nmax // 2 + 1)
        self.lib.o_heltrans(self.h, *[_ptr(x) for x in arrs], _ptr(Hk))
        return Hk

    def forcing_slow(self, timef, fstep, fold, fnew):
        """main3D.fpp's rand = 2 update: (1 - rmp) fold + rmp fnew."""
        fo = [self._c(x) for x in fold]
        fn = [self._c(x) for x in fnew]
        out = [self.czeros() for _ in range(3)]
        arr = lambda xs: (ctypes.c_void_p * 3)(*[x.ctypes.data for x in xs])
        self.lib.o_forcing_slow(self.h, int(timef), int(fstep), arr(fo), arr(fn), arr(out))
        return out

    def phaseshift(self, a, cdump):
        a = self._c(a).copy()
        self.lib.o_phaseshift(self.h, _ptr(a), cdump.real, cdump.imag)
        return a

    def vector3(self, a, b, c, d, e, f):
        arrs = [self._c(x) for x in (a, b, c, d, e, f)]
        out = [self.czeros() for _ in range(3)]
        self.lib.o_vector3(self.h, *[_ptr(x) for x in arrs], *[_ptr(x) for x in out])
        return out

    def nonlin3(self, a, b, c, d, e, f, dir):
        arrs = [self._c(x) for x in (a, b, c, d, e, f)]
        g = self.czeros()
        self.lib.o_nonlin3(self.h, *[_ptr(x) for x in arrs], _ptr(g), dir)
        return g

    def gauge3(self, a, b, c, dir):
        arrs = [self._c(x) for x in (a, b, c)]
        g = self.czeros()
        self.lib.o_gauge3(self.h, *[_ptr(x) for x in arrs], _ptr(g), dir)
        return g

    def mhd_run(self, nsteps, ord, dt, nu, mu, v, a, f=None, m=None):
        """nsteps RK steps of GHOST's MHD solver (mhd_rkstep2.f90)."""
        v = [self._c(x).copy() for x in v]
        a = [self._c(x).copy() for x in a]
        fp = [_ptr(self._c(x)) for x in f] if f is not None else [None] * 3
        mp = [_ptr(self._c(x)) for x in m] if m is not None else [None] * 3
        self.lib.o_mhd_run(self.h, nsteps, ord, dt, nu, mu, *[_ptr(x) for x in v], *[_ptr(x) for x in a], *fp, *mp)
        return v, a

    def phd_run(self, nsteps, ord, dt, nu, kappa, v, th, f=None, fs=None):
        """nsteps RK steps of GHOST's passive-scalar solver (phd_rkstep2.f90)."""
        v = [self._c(x).copy() for x in v]
        th = self._c(th).copy()
        fp = [_ptr(self._c(x)) for x in f] if f is not None else [None] * 3
        fsp = _ptr(self._c(fs)) if fs is not None else None
        self.lib.o_phd_run(self.h, nsteps, ord, dt, nu, kappa, *[_ptr(x) for x in v], _ptr(th), *fp, fsp)
        return v, th

    def variance(self, a, kin=1):
        return self.lib.o_variance(self.h, _ptr(self._c(a)), kin)

    def spectrscc(self, a, shift=0.0):
        Ek = np.zeros(self.nmax // 2 + 1)
        self.lib.o_spectrscc(self.h, _ptr(self._c(a)), shift, _ptr(Ek))
        return Ek

    def sctrans(self, a, b):
        Ek = np.zeros(self.nmax // 2 + 1)
        self.lib.o_sctrans(self.h, _ptr(self._c(a)), _ptr(self._c(b)), _ptr(Ek))
        return Ek

    def havgcomp(self, u, v, w, s, fo, bv, itype):
        """havgcomp: the horizontally averaged profile (nz,) of quantity itype."""
        arrs = [self._c(x) for x in (u, v, w, s)]
        gsh = np.zeros(self.nz)
        self.lib.o_havgcomp(self.h, *[_ptr(x) for x in arrs], fo, bv, itype, _ptr(gsh))
        return gsh

    def _an_nb(self, mode):
        return self.nz // 2 + 1 if mode == 0 else self.nmaxperp // 2 + 1

    def spec_aniso(self, mode, a, b, c, kin=1, hel=0):
        """specpara (mode 0) / specperp (mode 1): (3, nb) arrays of E and H."""
        a, b, c = self._c(a), self._c(b), self._c(c)
        nb = self._an_nb(mode)
        Ek, Hk = np.zeros(3 * nb), np.zeros(3 * nb)
        self.lib.o_spec_aniso(self.h, mode, _ptr(a), _ptr(b), _ptr(c), kin, hel, _ptr(Ek), _ptr(Hk))
        return Ek.reshape(3, nb), Hk.reshape(3, nb)

    def trans_aniso(self, mode, a, b, c, d, e, f, kin=1, curl=False):
        """entpara/entperp (curl False; kk2-weighted for kin 0), heltpara/heltperp (curl True)."""
        arrs = [self._c(x) for x in (a, b, c, d, e, f)]
        E = np.zeros(self._an_nb(mode))
        self.lib.o_trans_aniso(self.h, mode, *[_ptr(x) for x in arrs], int(kin == 0 and not curl), int(curl),
                               _ptr(E))
        return E

    def sharp(self, a, delta):
        a = self._c(a)
        b = self.czeros()
        self.lib.o_sharp(self.h, _ptr(a), _ptr(b), delta)
        return b

    # initial conditions -------------------------------------------------
    def random_vpot(self, seed, kdn, kup, shape):
        C = [self.czeros() for _ in range(3)]
        seed = self.lib.o_random_vpot(self.h, seed, kdn, kup, shape, *[_ptr(x) for x in C])
        return C, seed

    def random_solenoidal(self, seed, kdn, kup, shape, amp):
        v = [self.czeros() for _ in range(3)]
        seed = self.lib.o_random_solenoidal(self.h, seed, kdn, kup, shape, amp, *[_ptr(x) for x in v])
        return v, seed

    def abc(self, kdn, kup, A, B, C):
        R = [self.rzeros() for _ in range(3)]
        self.lib.o_abc(self.h, kdn, kup, A, B, C, *[_ptr(x) for x in R])
        return R

    def normalize(self, fx, fy, fz, f0, kin=1):
        fx, fy, fz = self._c(fx).copy(), self._c(fy).copy(), self._c(fz).copy()
        self.lib.o_normalize(self.h, _ptr(fx), _ptr(fy), _ptr(fz), f0, kin)
        return fx, fy, fz

    # RK -------------------------------------------------------------------
    def hd_rkstep2(self, o, dt, nu, v, C, f):
        v = [self._c(x).copy() for x in v]
        C = [self._c(x) for x in C]
        f = [self._c(x) for x in f]
        self.lib.o_hd_rkstep2(self.h, o, dt, nu, *[_ptr(x) for x in v], *[_ptr(x) for x in C],
                              *[_ptr(x) for x in f])
        return v

    def hd_run(self, nsteps, ord, dt, nu, v, f=None):
        v = [self._c(x).copy() for x in v]
        fp = [None, None, None] if f is None else [_ptr(self._c(x)) for x in f]
        fk = None if f is None else [self._c(x) for x in f]  # keep alive
        self.lib.o_hd_run(self.h, nsteps, ord, dt, nu, *[_ptr(x) for x in v],
                          *(fp if fk is None else [_ptr(x) for x in fk]))
        return v

    def advect3(self, a, b, c, d):
        a, b, c, d = self._c(a), self._c(b), self._c(c), self._c(d)
        e = self.czeros()
        self.lib.o_advect3(self.h, _ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(e))
        return e

    def bouss_run(self, nsteps, ord, dt, nu, kappa, omegaz, xmom, xtemp, v, th, f=None, fs=None):
        v = [self._c(x).copy() for x in v]
        th = self._c(th).copy()
        fk = None if f is None else [self._c(x) for x in f]
        fsk = None if fs is None else self._c(fs)
        self.lib.o_bouss_run(self.h, nsteps, ord, dt, nu, kappa, omegaz, xmom, xtemp,
                             *[_ptr(x) for x in v], _ptr(th),
                             *([None] * 3 if fk is None else [_ptr(x) for x in fk]),
                             None if fsk is None else _ptr(fsk))
        return v, th

    def set_kmax(self, kmax):
        self.lib.o_ctx_set_kmax(self.h, kmax)
        info = np.zeros(9)
        self.lib.o_ctx_info(self.h, info.ctypes.data)
        self.kmax = float(info[0])

    # EDQNM LES (pseudo/pseudospec3D_edqnm.f90, include/edqnmhd_rkstep2.f90) --
    def evedqnm(self, Eold, nu, time, kolmo=1.4):
        nb = self.nx // 2 + 1
        E = np.ascontiguousarray(Eold, dtype=np.float64)
        tepq, tve, Ext = np.zeros(nb), np.zeros(nb), np.zeros(3 * nb)
        self.lib.o_evedqnm(self.h, kolmo, _ptr(E), nu, time, _ptr(tepq), _ptr(tve), _ptr(Ext))
        return tepq, tve, Ext

    def evedqnm_h(self, Eold, Hold, nu, time, hel=1, kolmo=1.4):
        """evedqnm with helicity (pseudospec3D_edqnm.f90:24-92): returns
        tepq, thpq, tve, tvh [n/2+1] and the extrapolated Ext, Hxt [3(n/2+1)]."""
        nb = self.nx // 2 + 1
        E = np.ascontiguousarray(Eold, dtype=np.float64)
        H = np.ascontiguousarray(Hold, dtype=np.float64)
        out = [np.zeros(nb) for _ in range(4)] + [np.zeros(3 * nb), np.zeros(3 * nb)]
        self.lib.o_evedqnm_h(self.h, kolmo, _ptr(E), _ptr(H), nu, time, int(hel), *[_ptr(x) for x in out])
        return tuple(out)

    def edqnm_run(self, nsteps, ord, dt, nu, v, f=None, kolmo=1.4, t0=0.0, vcorrect=True, hel=0):
        v = [self._c(x).copy() for x in v]
        fk = None if f is None else [self._c(x) for x in f]
        if hel:
            self.lib.o_edqnm_run_h(self.h, nsteps, ord, dt, nu, kolmo, t0, int(vcorrect), int(hel),
                                   *[_ptr(x) for x in v], *([None] * 3 if fk is None else [_ptr(x) for x in fk]))
        else:
            self.lib.o_edqnm_run(self.h, nsteps, ord, dt, nu, kolmo, t0, int(vcorrect), *[_ptr(x) for x in v],
                                 *([None] * 3 if fk is None else [_ptr(x) for x in fk]))
        return v

    def vcorrect(self, v, ef, tepq, eold, dt):
        """vcorrect (heli = 0) of v with the per-mode energies ef of the step's start."""
        v = [self._c(x).copy() for x in v]
        ef = np.ascontiguousarray(ef, dtype=self.rdt)
        t = np.ascontiguousarray(tepq, dtype=np.float64)
        e = np.ascontiguousarray(eold, dtype=np.float64)
        self.lib.o_vcorrect(self.h, *[_ptr(x) for x in v], _ptr(ef), _ptr(t), _ptr(e), dt)
        return v

    def les_truncate(self, coarse: "Oracle", a, kc: int):
        """Modes |k| <= kc of this (fine) spectrum on the coarse grid, times (n/N)^3."""
        out = coarse.czeros()
        self.lib.o_les_truncate(self.h, coarse.h, _ptr(self._c(a)), _ptr(out), kc)
        return out

    def nthreads(self):
        return self.lib.o_nthreads()

    def set_threads(self, n):
        self.lib.o_set_threads(n)
