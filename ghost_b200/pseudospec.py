"""Host-side mirror of GHOST's fftp / pseudospec3D interface over the C ABI.

The names, argument order and meaning follow GHOST's Fortran routines
(3D/src/fftp-3/fftp3D.fpp, 3D/src/pseudo/pseudospec3D_hd.f90 and the HD /
ROTBOUSS include fragments): outputs are passed in, like Fortran INTENT(OUT)
arrays, and scalar results are returned.

Arrays are either CUDA tensors (torch; kept in HBM, no copies) or numpy
arrays (host; staged through the library's device buffers), with GHOST's
column-major layouts written as C-order shapes:
    spectral a(nz,ny,nx/2+1)  ->  shape (nx//2+1, ny, nz), complex
    real     r(nx,ny,nz)      ->  shape (nz, ny, nx), real
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GHOST_COMPLEX_TO_REAL, GHOST_DOUBLE, GHOST_REAL_TO_COMPLEX, GHOST_SINGLE, check

try:  # torch is only needed for device arrays
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_tensor(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor)


@dataclass
class FFTPlan:
    """fftp3d_create_plan's FFTPLAN (fftp-3/fftp_mod.fpp)."""
    handle: ctypes.c_void_p
    n: tuple
    fftdir: int


class Ghost:
    """One GHOST grid: the grid/kes/ali/boxsize module state plus the HD
    routines, executed by libghost_b200 on the current CUDA device."""

    def __init__(self, nx: int, ny: int | None = None, nz: int | None = None,
                 Lx: float = 1.0, Ly: float = 1.0, Lz: float = 1.0, arbsize: bool = False,
                 precision: str = "fp64", stream=None, nruns: int = 1, handle=None):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.lib = _lib.load()
        self.precision = precision
        self.nruns = nruns
        self.owned = handle is None
        code = {"fp32": GHOST_SINGLE, "fp64": GHOST_DOUBLE}[precision]
        h = ctypes.c_void_p()
        if handle is not None:
            h = handle
        elif nruns > 1:
            check(self.lib.ghost_ctx_create_batch(nx, ny, nz, nruns, code, ctypes.byref(h)), "ghost_ctx_create_batch")
        else:
            check(self.lib.ghost_ctx_create(nx, ny, nz, Lx, Ly, Lz, int(bool(arbsize)), code, ctypes.byref(h)),
                  "ghost_ctx_create")
        self.h = h
        info = _lib.GhostInfo()
        check(self.lib.ghost_ctx_get_info(self.h, ctypes.byref(info)), "ghost_ctx_get_info")
        self.info = info
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nxh = nx // 2 + 1
        self.kmax, self.tiny, self.nmax, self.Dkk = info.kmax, info.tiny, info.nmax, info.Dkk
        self.nmaxperp = info.nmaxperp
        self.rdtype_np = np.float32 if precision == "fp32" else np.float64
        self.cdtype_np = np.complex64 if precision == "fp32" else np.complex128
        if stream is None and handle is None and torch is not None and torch.cuda.is_available():
            stream = torch.cuda.current_stream().cuda_stream
        if stream is not None:
            check(self.lib.ghost_ctx_set_stream(self.h, ctypes.c_void_p(stream)), "ghost_ctx_set_stream")
        self.stream = stream

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "owned", True):
                self.lib.ghost_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------
    @property
    def sshape(self):
        return (self.nxh * self.nruns, self.ny, self.nz)

    @property
    def rshape(self):
        return (self.nz, self.ny, self.nx)

    @property
    def ctorch(self):
        return torch.complex64 if self.precision == "fp32" else torch.complex128

    @property
    def rtorch(self):
        return torch.float32 if self.precision == "fp32" else torch.float64

    def czeros(self, device="cuda"):
        return torch.zeros(self.sshape, dtype=self.ctorch, device=device)

    def rzeros(self, device="cuda"):
        return torch.zeros(self.rshape, dtype=self.rtorch, device=device)

    def _ptr(self, x, kind: str):
        if x is None:
            return None
        shape = self.sshape if kind == "c" else self.rshape
        if _is_tensor(x):
            want = self.ctorch if kind == "c" else self.rtorch
            if x.dtype != want or tuple(x.shape) != shape or not x.is_contiguous():
                raise ValueError(f"expected contiguous {want} {shape}, got {x.dtype} {tuple(x.shape)}")
            return ctypes.c_void_p(x.data_ptr())
        if isinstance(x, np.ndarray):
            want = self.cdtype_np if kind == "c" else self.rdtype_np
            if x.dtype != want or x.shape != shape or not x.flags["C_CONTIGUOUS"]:
                raise ValueError(f"expected C-contiguous {np.dtype(want)} {shape}, got {x.dtype} {x.shape}")
            return ctypes.c_void_p(x.ctypes.data)
        raise TypeError(f"unsupported array type {type(x)}")

    def entrans(self, a, b, c, d, e, f, kin: int = 1):
        """entrans: GHOST's Ektot, the shell-binned transfer Re(v . conj(nl))."""
        Ek = np.zeros(self.nmax // 2 + 1)
        check(self.lib.ghost_entrans(self.h, *[self._ptr(x, "c") for x in (a, b, c, d, e, f)], kin,
                                     Ek.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_entrans")
        return Ek

    def heltrans(self, a, b, c, d, e, f, kin: int = 1):
        """heltrans: GHOST's Hktot, the shell-binned Re(curl v . conj(nl))."""
        Hk = np.zeros(self.nmax // 2 + 1)
        check(self.lib.ghost_heltrans(self.h, *[self._ptr(x, "c") for x in (a, b, c, d, e, f)], kin,
                                      Hk.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_heltrans")
        return Hk

    def forcing_slow(self, timef: int, fstep: int, fold, fnew, f):
        """GHOST's rand = 2 forcing: f = (1 - rmp) fold + rmp fnew, rmp = (timef+1)/fstep."""
        check(self.lib.ghost_forcing_slow(self.h, int(timef), int(fstep), *[self._ptr(x, "c") for x in fold],
                                          *[self._ptr(x, "c") for x in fnew], *[self._ptr(x, "c") for x in f]),
              "forcing_slow")

    def phaseshift(self, a, cdump: complex):
        """phaseshift: a *= cdump in place (conj on the kx = 0 mirror half)."""
        check(self.lib.ghost_phaseshift(self.h, self._ptr(a, "c"), cdump.real, cdump.imag), "phaseshift")

    # ---- MHD (MHD_SOL)
    def vector3(self, a, b, c, d, e, f, x=None, y=None, z=None):
        out = [self.czeros() if o is None else o for o in (x, y, z)]
        check(self.lib.ghost_vector3(self.h, *[self._ptr(q, "c") for q in (a, b, c, d, e, f, *out)]), "vector3")
        return out

    def nonlin3(self, a, b, c, d, e, f, dir: int, g=None):
        g = self.czeros() if g is None else g
        check(self.lib.ghost_nonlin3(self.h, *[self._ptr(q, "c") for q in (a, b, c, d, e, f, g)], dir), "nonlin3")
        return g

    def gauge3(self, a, b, c, dir: int, g=None):
        g = self.czeros() if g is None else g
        check(self.lib.ghost_gauge3(self.h, *[self._ptr(q, "c") for q in (a, b, c, g)], dir), "gauge3")
        return g

    def mhd_run(self, nsteps, ord, dt, nu, mu, vx, vy, vz, ax, ay, az, f=(None, None, None), m=(None, None, None)):
        check(self.lib.ghost_mhd_run(self.h, nsteps, ord, dt, nu, mu,
                                     *[self._ptr(q, "c") for q in (vx, vy, vz, ax, ay, az, *f, *m)]), "mhd_run")

    # ---- passive scalar (PHD_SOL)
    def phd_run(self, nsteps, ord, dt, nu, kappa, vx, vy, vz, th, fx=None, fy=None, fz=None, fs=None):
        check(self.lib.ghost_phd_run(self.h, nsteps, ord, dt, nu, kappa,
                                     *[self._ptr(x, "c") for x in (vx, vy, vz, th, fx, fy, fz, fs)]), "phd_run")

    def variance(self, a, kin: int = 1) -> float:
        out = ctypes.c_double()
        check(self.lib.ghost_variance(self.h, self._ptr(a, "c"), kin, ctypes.byref(out)), "ghost_variance")
        return out.value

    def spectrscc(self, a, shift: float = 0.0):
        Ek = np.zeros(self.nmax // 2 + 1)
        check(self.lib.ghost_spectrscc(self.h, self._ptr(a, "c"), shift,
                                       Ek.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_spectrscc")
        return Ek

    def sctrans(self, a, b, isc: int = 0):
        Ek = np.zeros(self.nmax // 2 + 1)
        check(self.lib.ghost_sctrans(self.h, self._ptr(a, "c"), self._ptr(b, "c"), isc,
                                     Ek.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_sctrans")
        return Ek

    def havgcomp(self, u, v, w, s, fo: float, bv: float, itype: int):
        """havgcomp: the horizontally averaged profile (nz,) of quantity itype."""
        gsh = np.zeros(self.nz)
        check(self.lib.ghost_havgcomp(self.h, *[self._ptr(x, "c") for x in (u, v, w, s)], fo, bv, itype,
                                      gsh.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_havgcomp")
        return gsh

    def tbouss(self, u, v, w, s, fo: float, bv: float):
        """tbouss: (avg, max, min) over z of the 11 havgcomp profiles."""
        out = [np.zeros(11) for _ in range(3)]
        PDt = ctypes.POINTER(ctypes.c_double)
        check(self.lib.ghost_tbouss(self.h, *[self._ptr(x, "c") for x in (u, v, w, s)], fo, bv,
                                    *[o.ctypes.data_as(PDt) for o in out]), "ghost_tbouss")
        return tuple(out)

    def _aniso_nb(self, para: bool) -> int:
        return self.nz // 2 + 1 if para else self.nmaxperp // 2 + 1

    def _spec_aniso(self, fn, para, a, b, c, kin, hel):
        nb = self._aniso_nb(para)
        Ek, Hk = np.zeros(3 * nb), np.zeros(3 * nb)
        PDt = ctypes.POINTER(ctypes.c_double)
        check(getattr(self.lib, fn)(self.h, *[self._ptr(x, "c") for x in (a, b, c)], kin, hel,
                                    Ek.ctypes.data_as(PDt), Hk.ctypes.data_as(PDt)), fn)
        return Ek.reshape(3, nb), Hk.reshape(3, nb)

    def specpara(self, a, b, c, kin: int = 1, hel: int = 0):
        """specpara: (3, nz/2+1) arrays (total, horizontal, vertical) of E and H."""
        return self._spec_aniso("ghost_specpara", True, a, b, c, kin, hel)

    def specperp(self, a, b, c, kin: int = 1, hel: int = 0):
        """specperp: (3, nmaxperp/2+1) arrays (total, kz=0 horizontal, kz=0 vertical)."""
        return self._spec_aniso("ghost_specperp", False, a, b, c, kin, hel)

    def _trans_aniso(self, fn, para, fields, kin):
        out = np.zeros(self._aniso_nb(para))
        check(getattr(self.lib, fn)(self.h, *[self._ptr(x, "c") for x in fields], kin,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), fn)
        return out

    def entpara(self, a, b, c, d, e, f, kin: int = 1):
        return self._trans_aniso("ghost_entpara", True, (a, b, c, d, e, f), kin)

    def entperp(self, a, b, c, d, e, f, kin: int = 1):
        return self._trans_aniso("ghost_entperp", False, (a, b, c, d, e, f), kin)

    def heltpara(self, a, b, c, d, e, f, kin: int = 1):
        return self._trans_aniso("ghost_heltpara", True, (a, b, c, d, e, f), kin)

    def heltperp(self, a, b, c, d, e, f, kin: int = 1):
        return self._trans_aniso("ghost_heltperp", False, (a, b, c, d, e, f), kin)

    # ---- GHOST's binary field files (mpiio/binary_io.f90)
    def io_write(self, real, path: str, swap: bool = False):
        """io_write: a real field (nz, ny, nx), x fastest, to a raw GP file."""
        check(self.lib.ghost_io_write(self.h, self._ptr(real, "r"), os.fsencode(path), int(swap)), "ghost_io_write")

    def io_read(self, path: str, out=None, swap: bool = False):
        """io_read: a raw GP file of nx*ny*nz values into a real field."""
        out = self.rzeros() if out is None else out
        check(self.lib.ghost_io_read(self.h, os.fsencode(path), int(swap), self._ptr(out, "r")), "ghost_io_read")
        return out

    def io_output(self, spec, path: str, swap: bool = False):
        """One field of GHOST's output step: the real field of spec/(nx ny nz)."""
        check(self.lib.ghost_io_output(self.h, self._ptr(spec, "c"), os.fsencode(path), int(swap)), "ghost_io_output")

    def io_restart(self, path: str, out=None, swap: bool = False):
        """One field of GHOST's restart: io_read, then the forward transform."""
        out = self.czeros() if out is None else out
        check(self.lib.ghost_io_restart(self.h, os.fsencode(path), int(swap), self._ptr(out, "c")), "ghost_io_restart")
        return out

    def set_tile_cfg(self, cfg: int):
        check(self.lib.ghost_ctx_set_tile_cfg(self.h, int(cfg)), "ghost_ctx_set_tile_cfg")

    def tile_cfg(self) -> int:
        c = ctypes.c_int()
        check(self.lib.ghost_ctx_get_tile_cfg(self.h, ctypes.byref(c)), "ghost_ctx_get_tile_cfg")
        return c.value

    def hd_autotune(self, ord: int, dt: float, nu: float, vx, vy, vz, fx=None, fy=None, fz=None) -> int:
        """Pick the fastest tile variant for this run (v does not advance)."""
        c = ctypes.c_int()
        check(self.lib.ghost_hd_autotune(self.h, ord, dt, nu, *[self._ptr(x, "c") for x in (vx, vy, vz, fx, fy, fz)],
                                         ctypes.byref(c)), "ghost_hd_autotune")
        return c.value

    def launch_count(self) -> int:
        n = ctypes.c_longlong()
        check(self.lib.ghost_ctx_launch_count(self.h, ctypes.byref(n)), "ghost_ctx_launch_count")
        return n.value

    def enable_timers(self, on: bool = True):
        check(self.lib.ghost_ctx_enable_timers(self.h, int(on)), "ghost_ctx_enable_timers")

    def read_timers(self) -> dict:
        """{kernel kind: (milliseconds, launches)} since the last read."""
        n = len(_lib.TIMER_NAMES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        check(self.lib.ghost_ctx_read_timers(self.h, ms, cnt), "ghost_ctx_read_timers")
        return {name: (ms[k], cnt[k]) for k, name in enumerate(_lib.TIMER_NAMES) if cnt[k]}

    def synchronize(self):
        check(self.lib.ghost_ctx_synchronize(self.h), "ghost_ctx_synchronize")

    def inject_stall(self, on: bool):
        """Fault injection: pipelined passes wait on a barrier nothing completes."""
        check(self.lib.ghost_ctx_inject_stall(self.h, int(on)), "ghost_ctx_inject_stall")

    def set_wait_cap(self, cap: int):
        """Bound on device-side polls of every pipelined wait (0: default)."""
        check(self.lib.ghost_ctx_set_wait_cap(self.h, cap), "ghost_ctx_set_wait_cap")

    def set_kmax(self, kmax: float):
        check(self.lib.ghost_ctx_set_kmax(self.h, kmax), "ghost_ctx_set_kmax")
        info = _lib.GhostInfo()
        check(self.lib.ghost_ctx_get_info(self.h, ctypes.byref(info)), "ghost_ctx_get_info")
        self.kmax = info.kmax

    # ---------------------------------------------------------------- fftp
    def fftp3d_create_plan(self, n, fftdir: int, flags: int = 0) -> FFTPlan:
        arr = (ctypes.c_int * 3)(*n)
        h = ctypes.c_void_p()
        check(self.lib.ghost_fftp3d_create_plan(self.h, arr, fftdir, flags, ctypes.byref(h)),
              "fftp3d_create_plan")
        return FFTPlan(h, tuple(n), fftdir)

    def fftp3d_destroy_plan(self, plan: FFTPlan):
        check(self.lib.ghost_fftp3d_destroy_plan(plan.handle), "fftp3d_destroy_plan")

    def fftp3d_real_to_complex(self, plan: FFTPlan, inp, out):
        check(self.lib.ghost_fftp3d_real_to_complex(plan.handle, self._ptr(inp, "r"), self._ptr(out, "c")),
              "fftp3d_real_to_complex")

    def fftp3d_complex_to_real(self, plan: FFTPlan, inp, out):
        check(self.lib.ghost_fftp3d_complex_to_real(plan.handle, self._ptr(inp, "c"), self._ptr(out, "r")),
              "fftp3d_complex_to_real")

    # --------------------------------------------------- pseudospec3D_hd
    def derivk3(self, a, b, dir: int):
        check(self.lib.ghost_derivk3(self.h, self._ptr(a, "c"), self._ptr(b, "c"), dir), "derivk3")

    def laplak3(self, a, b):
        check(self.lib.ghost_laplak3(self.h, self._ptr(a, "c"), self._ptr(b, "c")), "laplak3")

    def rotor3(self, a, b, c, dir: int):
        check(self.lib.ghost_rotor3(self.h, self._ptr(a, "c"), self._ptr(b, "c"), self._ptr(c, "c"), dir),
              "rotor3")

    def prodre3(self, a, b, c, d, e, f):
        check(self.lib.ghost_prodre3(self.h, *[self._ptr(x, "c") for x in (a, b, c, d, e, f)]), "prodre3")

    def nonlhd3(self, a, b, c, g, dir: int):
        check(self.lib.ghost_nonlhd3(self.h, *[self._ptr(x, "c") for x in (a, b, c, g)], dir), "nonlhd3")

    def energy(self, a, b, c, kin: int) -> float:
        d = ctypes.c_double()
        check(self.lib.ghost_energy(self.h, *[self._ptr(x, "c") for x in (a, b, c)], ctypes.byref(d), kin),
              "energy")
        return d.value

    def helicity(self, a, b, c) -> float:
        d = ctypes.c_double()
        check(self.lib.ghost_helicity(self.h, *[self._ptr(x, "c") for x in (a, b, c)], ctypes.byref(d)),
              "helicity")
        return d.value

    def cross(self, a, b, c, d, e, f, kin: int) -> float:
        g = ctypes.c_double()
        check(self.lib.ghost_cross(self.h, *[self._ptr(x, "c") for x in (a, b, c, d, e, f)], ctypes.byref(g),
                                   kin), "cross")
        return g.value

    def divergence(self, a, b, c) -> float:
        d = ctypes.c_double()
        check(self.lib.ghost_divergence(self.h, *[self._ptr(x, "c") for x in (a, b, c)], ctypes.byref(d)),
              "divergence")
        return d.value

    def maxabs(self, a, b, c, kin: int) -> float:
        d = ctypes.c_double()
        check(self.lib.ghost_maxabs(self.h, *[self._ptr(x, "c") for x in (a, b, c)], ctypes.byref(d), kin),
              "maxabs")
        return d.value

    def spectrumc(self, a, b, c, kin: int = 1, hel: int = 0):
        nb = self.nmax // 2 + 1
        Ek = np.zeros(nb)
        Hk = np.zeros(nb)
        pd = ctypes.POINTER(ctypes.c_double)
        check(self.lib.ghost_spectrumc(self.h, *[self._ptr(x, "c") for x in (a, b, c)], kin, hel,
                                       Ek.ctypes.data_as(pd), Hk.ctypes.data_as(pd)), "spectrumc")
        return Ek, Hk

    def hdcheck(self, vx, vy, vz, fx, fy, fz, hel: int = 1, chk: int = 0):
        out = np.zeros(5)
        check(self.lib.ghost_hdcheck(self.h, *[self._ptr(x, "c") for x in (vx, vy, vz, fx, fy, fz)], hel, chk,
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "hdcheck")
        return {"eng": out[0], "ens": out[1], "khe": out[2], "pot": out[3], "div": out[4]}

    def normalize(self, fx, fy, fz, f0: float, kin: int = 1):
        check(self.lib.ghost_normalize(self.h, *[self._ptr(x, "c") for x in (fx, fy, fz)], f0, kin), "normalize")

    def sharp(self, a, b, delta: float):
        check(self.lib.ghost_sharp(self.h, self._ptr(a, "c"), self._ptr(b, "c"), delta), "sharp")

    # -------------------------------------------------------------- RK
    def hd_rkstep1(self, vx, vy, vz, C1, C2, C3):
        check(self.lib.ghost_hd_rkstep1(self.h, *[self._ptr(x, "c") for x in (vx, vy, vz, C1, C2, C3)]),
              "hd_rkstep1")

    def hd_rkstep2(self, o: int, dt: float, nu: float, vx, vy, vz, C1, C2, C3, fx=None, fy=None, fz=None):
        check(self.lib.ghost_hd_rkstep2(self.h, o, dt, nu,
                                        *[self._ptr(x, "c") for x in (vx, vy, vz, C1, C2, C3, fx, fy, fz)]),
              "hd_rkstep2")

    def hd_run(self, nsteps: int, ord: int, dt: float, nu: float, vx, vy, vz, fx=None, fy=None, fz=None,
               C=(None, None, None)):
        check(self.lib.ghost_hd_run(self.h, nsteps, ord, dt, nu,
                                    *[self._ptr(x, "c") for x in (vx, vy, vz, *C, fx, fy, fz)]), "hd_run")

    # ------------------------------------------------------- Boussinesq
    def advect3(self, a, b, c, d, e):
        check(self.lib.ghost_advect3(self.h, *[self._ptr(x, "c") for x in (a, b, c, d, e)]), "advect3")

    def bouss_rkstep2(self, o, dt, nu, kappa, omegaz, xmom, xtemp, vx, vy, vz, th, C1, C2, C3, C20,
                      fx=None, fy=None, fz=None, fs=None):
        check(self.lib.ghost_bouss_rkstep2(
            self.h, o, dt, nu, kappa, omegaz, xmom, xtemp,
            *[self._ptr(x, "c") for x in (vx, vy, vz, th, C1, C2, C3, C20, fx, fy, fz, fs)]), "bouss_rkstep2")

    def bouss_run(self, nsteps, ord, dt, nu, kappa, omegaz, xmom, xtemp, vx, vy, vz, th,
                  fx=None, fy=None, fz=None, fs=None):
        check(self.lib.ghost_bouss_run(
            self.h, nsteps, ord, dt, nu, kappa, omegaz, xmom, xtemp,
            *[self._ptr(x, "c") for x in (vx, vy, vz, th, fx, fy, fz, fs)]), "bouss_run")

    # ------------------------------------------------------------ ICs
    def init_random_solenoidal(self, seed: int, kdn: float, kup: float, shape: int, amp: float, ox, oy, oz) -> int:
        s = ctypes.c_int32(seed)
        check(self.lib.ghost_init_random_solenoidal(self.h, ctypes.byref(s), kdn, kup, shape, amp,
                                                    *[self._ptr(x, "c") for x in (ox, oy, oz)]),
              "init_random_solenoidal")
        return s.value


    # ------------------------------------------------------- batches
    def batch_set_nu(self, nu):
        arr = np.ascontiguousarray(nu, dtype=np.float64)
        check(self.lib.ghost_batch_set_nu(self.h, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              "ghost_batch_set_nu")

    def batch_energy(self, a, b, c, kin: int = 1):
        out = np.zeros(self.nruns)
        check(self.lib.ghost_batch_energy(self.h, *[self._ptr(x, "c") for x in (a, b, c)], kin,
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_batch_energy")
        return out

    def batch_init_random_solenoidal(self, seeds, kdn, kup, shape, amp, ox, oy, oz):
        arr = (ctypes.c_int32 * self.nruns)(*seeds)
        check(self.lib.ghost_batch_init_random_solenoidal(self.h, arr, kdn, kup, shape, amp,
                                                          *[self._ptr(x, "c") for x in (ox, oy, oz)]),
              "ghost_batch_init_random_solenoidal")
        return list(arr)


class Ensemble:
    """Batches of cubic runs of several sizes advanced together: one batched
    context per size class, one RK step of all classes replayed as a CUDA
    graph (ghost_ensemble_* of the C ABI)."""

    def __init__(self, sizes, nruns, precision: str = "fp32"):
        self.lib = _lib.load()
        self.sizes, self.nruns, self.precision = list(sizes), list(nruns), precision
        code = {"fp32": GHOST_SINGLE, "fp64": GHOST_DOUBLE}[precision]
        h = ctypes.c_void_p()
        n = (ctypes.c_int * len(sizes))(*sizes)
        r = (ctypes.c_int * len(sizes))(*nruns)
        check(self.lib.ghost_ensemble_create(len(sizes), n, r, code, ctypes.byref(h)), "ghost_ensemble_create")
        self.h = h
        self.total = sum(nruns)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ghost_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, seeds, nu, kdn=1.0, kup_frac=1.0 / 3.0, shape=1, amp=1.0):
        s = (ctypes.c_int32 * self.total)(*seeds)
        v = np.ascontiguousarray(nu, dtype=np.float64)
        check(self.lib.ghost_ensemble_init(self.h, s, kdn, kup_frac, shape, amp,
                                           v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "ghost_ensemble_init")

    def autotune(self, ord: int, dt: float):
        cfg = (ctypes.c_int * len(self.sizes))()
        check(self.lib.ghost_ensemble_autotune(self.h, ord, dt, cfg), "ghost_ensemble_autotune")
        return list(cfg)

    def run(self, nsteps: int, ord: int, dt: float):
        check(self.lib.ghost_ensemble_run(self.h, nsteps, ord, dt), "ghost_ensemble_run")

    def set_mode(self, multi: bool):
        """True: each pass one launch over every class; False: per-class launches on per-class streams."""
        check(self.lib.ghost_ensemble_set_mode(self.h, int(bool(multi))), "ghost_ensemble_set_mode")

    def mode(self) -> bool:
        m = ctypes.c_int()
        check(self.lib.ghost_ensemble_get_mode(self.h, ctypes.byref(m)), "ghost_ensemble_get_mode")
        return bool(m.value)

    def energy(self, kin: int = 1):
        out = np.zeros(self.total)
        check(self.lib.ghost_ensemble_energy(self.h, kin, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              "ghost_ensemble_energy")
        return out

    def fields(self, c: int):
        """Class c's batched velocity as CUDA tensors (nruns*(n/2+1), n, n)."""
        ptr = [ctypes.c_void_p() for _ in range(3)]
        check(self.lib.ghost_ensemble_fields(self.h, c, *[ctypes.byref(p) for p in ptr]), "ghost_ensemble_fields")
        n, r = self.sizes[c], self.nruns[c]
        shape = (r * (n // 2 + 1), n, n)
        dt = torch.complex64 if self.precision == "fp32" else torch.complex128
        return [_tensor_view(p.value, shape, dt) for p in ptr]

    def class_ctx(self, c: int) -> Ghost:
        h = ctypes.c_void_p()
        check(self.lib.ghost_ensemble_class(self.h, c, ctypes.byref(h)), "ghost_ensemble_class")
        n = self.sizes[c]
        return Ghost(n, precision=self.precision, nruns=self.nruns[c], handle=h)


def _tensor_view(ptr: int, shape, dtype):
    """A CUDA tensor aliasing library-owned device memory (no copy)."""
    class _Arr:
        __cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": "<c8" if dtype == torch.complex64 else "<c16",
            "data": (ptr, False), "version": 3, "strides": None}
    return torch.as_tensor(_Arr(), device="cuda")


__all__ = ["Ghost", "Ensemble", "FFTPlan", "GHOST_REAL_TO_COMPLEX", "GHOST_COMPLEX_TO_REAL"]


def io_filename(dir: str, name: str, index: int, width: int = 4) -> str:
    """GHOST's field file name "<dir>/<name>.NNNN.out" (fmtext '(i4.4)')."""
    buf = ctypes.create_string_buffer(4096)
    check(_lib.load().ghost_io_filename(os.fsencode(dir), os.fsencode(name), index, width, buf, len(buf)),
          "ghost_io_filename")
    return os.fsdecode(buf.value)
