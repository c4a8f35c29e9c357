"""Slab decomposition of one HD run over ranks, in GHOST's MPI layout.

GHOST splits the spectral fields into kx-slabs (rows ista..iend of
1..nx/2+1) and the real fields into z-slabs (planes ksta..kend of 1..nz),
both by range() (fftp-3/fftp.f90; main3D.fpp:634-635), and every 3D
transform moves data between the two layouts with one all-to-all
(fftp-3/fftp3D.fpp:158-201, 255-278, 434-488).  Here one HD substep
(include/hd_rkstep2.f90) on rank r is

    front (Z and Y inverse of v and curl v on the kx-slab, 6 fields)
    -> pack -> all-to-all -> unpack        (kx-slab -> z-slab)
    -> x pass (omega x v in real space, x transforms; 6 -> 3 fields)
    -> pack -> all-to-all -> unpack        (z-slab -> kx-slab)
    -> back (Y and Z forward, truncated update of v on the kx-slab).

The local passes, the packing and the unpacking are the library's
(ghost_slab_* in libghost_b200); the all-to-all is
torch.distributed.all_to_all_single on the default process group (one
process per GPU over NCCL) in Slab.run, or device copies between the
ranks that one process holds in run_local.  Fields are torch tensors on
the device: a rank's kx-slab of a spectral field is (nxh_loc, ny, nz),
Fortran (nz, ny, ista:iend).  Every substep after the first of a run is
zero-pruned as in ghost_hd_run: pruned passes, and exchanges of the kx
rows below Slab.rows only.
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import GHOST_DOUBLE, GHOST_SINGLE, check

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def slab_range(n1: int, n2: int, nprocs: int, irank: int) -> tuple[int, int]:
    """GHOST's range(n1,n2,nprocs,irank,ista,iend) (fftp-3/fftp.f90):
    1-based inclusive bounds of rank irank's share of n1..n2."""
    lib = _lib.load()
    a, b = ctypes.c_int(), ctypes.c_int()
    check(lib.ghost_slab_range(n1, n2, nprocs, irank, ctypes.byref(a), ctypes.byref(b)), "ghost_slab_range")
    return a.value, b.value


def slab_layout(nx: int, nz: int, nranks: int):
    """Per-rank 0-based kx-row starts and counts, z-plane starts and counts."""
    ista, nxhl, ksta, nzl = [], [], [], []
    for r in range(nranks):
        a, b = slab_range(1, nx // 2 + 1, nranks, r)
        ka, kb = slab_range(1, nz, nranks, r)
        ista.append(a - 1)
        nxhl.append(b - a + 1)
        ksta.append(ka - 1)
        nzl.append(kb - ka + 1)
    return ista, nxhl, ksta, nzl


def live_rows(ista, nxhl, rows):
    """kx rows of every rank that a pruned exchange moves: the prefix of its
    slab below the global live rows (None: every row)."""
    if rows is None:
        return list(nxhl)
    return [max(0, min(rows - a, n)) for a, n in zip(ista, nxhl)]


def exchange_counts(nxhl, nzl, ny: int, rank: int, direction: int, nf: int):
    """Complex values sent to and received from every peer by `rank` in one
    all-to-all of nf fields.  Direction 0 (kx-slab -> z-slab): the chunk
    for peer p is nf blocks of my kx rows x ny x p's z planes; the chunk
    from p is nf blocks of p's rows x ny x my planes.  Direction 1 is the
    reverse.  For a pruned exchange nxhl is the ranks' live rows."""
    n = len(nxhl)
    mine = [nf * nxhl[rank] * ny * nzl[p] for p in range(n)]
    theirs = [nf * nxhl[p] * ny * nzl[rank] for p in range(n)]
    return (mine, theirs) if direction == 0 else (theirs, mine)


def all_to_all(recv, send, recv_counts, send_counts, group=None):
    """One all-to-all of complex buffers (peer-major chunks of the given
    counts) over torch.distributed; the buffers travel as their real
    and imaginary parts."""
    import torch.distributed as dist
    r = torch.view_as_real(recv[:sum(recv_counts)]).reshape(-1)
    s = torch.view_as_real(send[:sum(send_counts)]).reshape(-1)
    dist.all_to_all_single(r, s, [2 * c for c in recv_counts], [2 * c for c in send_counts], group=group)


class Slab:
    """One rank's share of a slab-decomposed HD run: the library's slab
    context and the work arrays of the substep."""

    def __init__(self, nx: int, ny: int | None = None, nz: int | None = None, Lx: float = 1.0, Ly: float = 1.0,
                 Lz: float = 1.0, arbsize: bool = False, precision: str = "fp64", rank: int = 0, nranks: int = 1,
                 stream=None):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.lib = _lib.load()
        self.nx, self.ny, self.nz, self.nxh = nx, ny, nz, nx // 2 + 1
        self.rank, self.nranks, self.precision = rank, nranks, precision
        code = {"fp32": GHOST_SINGLE, "fp64": GHOST_DOUBLE}[precision]
        h = ctypes.c_void_p()
        check(self.lib.ghost_slab_create(nx, ny, nz, Lx, Ly, Lz, int(bool(arbsize)), code, rank, nranks,
                                         ctypes.byref(h)), "ghost_slab_create")
        self.h = h
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        check(self.lib.ghost_slab_set_stream(self.h, ctypes.c_void_p(stream)), "ghost_slab_set_stream")
        self.ista, self.nxhl, self.ksta, self.nzl = slab_layout(nx, nz, nranks)
        rows = ctypes.c_int()
        check(self.lib.ghost_slab_rows(self.h, ctypes.byref(rows)), "ghost_slab_rows")
        self.rows = rows.value
        self.kshape = (self.nxhl[rank], ny, nz)
        self.zshape = (self.nxh, ny, self.nzl[rank])
        dt = torch.complex64 if precision == "fp32" else torch.complex128
        dev = torch.device("cuda", torch.cuda.current_device())
        self.w = [torch.zeros(self.kshape, dtype=dt, device=dev) for _ in range(6)]   # kx-slab work fields
        self.z = [torch.zeros(self.zshape, dtype=dt, device=dev) for _ in range(6)]   # z-slab work fields
        self.C = [torch.zeros(self.kshape, dtype=dt, device=dev) for _ in range(3)]   # RK copy (hd_rkstep1)
        # (direction, pruned) -> (send counts, receive counts)
        self.counts = {(d, pr): exchange_counts(live_rows(self.ista, self.nxhl, self.rows if pr else None), self.nzl,
                                                ny, rank, d, 6 if d == 0 else 3)
                       for d in (0, 1) for pr in (False, True)}
        nsend = max(sum(self.counts[d, False][0]) for d in (0, 1))
        nrecv = max(sum(self.counts[d, False][1]) for d in (0, 1))
        self.send = torch.empty(nsend, dtype=dt, device=dev)
        self.recv = torch.empty(nrecv, dtype=dt, device=dev)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ghost_slab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch_count(self) -> int:
        """Kernels launched by this rank's slab contexts so far."""
        n = ctypes.c_longlong()
        check(self.lib.ghost_slab_launch_count(self.h, ctypes.byref(n)), "ghost_slab_launch_count")
        return n.value

    @staticmethod
    def _pp(ts):
        return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])

    def _fields(self, v):
        for t in v:
            if tuple(t.shape) != self.kshape or not t.is_cuda or not t.is_contiguous():
                raise ValueError(f"slab fields must be contiguous device arrays of shape {self.kshape}")
        return v

    # -- the phases of one substep ------------------------------------
    def front(self, v, copy: bool, prune: bool = False):
        check(self.lib.ghost_slab_hd_front(self.h, self._pp(self._fields(v)), self._pp(self.C), int(copy), int(prune),
                                           self._pp(self.w)), "ghost_slab_hd_front")

    def pack(self, direction: int, prune: bool = False):
        fields = self.w if direction == 0 else self.z[:3]
        check(self.lib.ghost_slab_pack(self.h, direction, len(fields), int(prune), self._pp(fields),
                                       ctypes.c_void_p(self.send.data_ptr())), "ghost_slab_pack")

    def unpack(self, direction: int, prune: bool = False):
        fields = self.z if direction == 0 else self.w[:3]
        check(self.lib.ghost_slab_unpack(self.h, direction, len(fields), int(prune),
                                         ctypes.c_void_p(self.recv.data_ptr()), self._pp(fields)), "ghost_slab_unpack")

    def xpass(self, prune: bool = False):
        # one rank: the kx-slab is the whole field and the z-slab layout is the same, so the x pass
        # runs on the front's output in place and no exchange is needed
        z = self.w if self.nranks == 1 else self.z
        check(self.lib.ghost_slab_hd_xpass(self.h, int(prune), self._pp(z), self._pp(z[:3])), "ghost_slab_hd_xpass")

    def back(self, o: int, dt: float, nu: float, v, f=None, prune: bool = False):
        fp = self._pp(self._fields(f)) if f is not None else None
        check(self.lib.ghost_slab_hd_back(self.h, o, dt, nu, int(prune), self._pp(self.w[:3]),
                                          self._pp(self._fields(v)), self._pp(self.C), fp), "ghost_slab_hd_back")

    # -- runs -----------------------------------------------------------
    def run(self, nsteps: int, ord: int, dt: float, nu: float, vx, vy, vz, fx=None, fy=None, fz=None, group=None,
            exchange_events=None):
        """nsteps RK steps of order ord (GHOST's RK loop, main3D.fpp:3195-3231)
        of this rank's kx-slab of v, the transposes as NCCL all-to-alls.
        Every substep after the first is zero-pruned, as in ghost_hd_run.
        exchange_events: a list to which CUDA event pairs bracketing each
        all-to-all (on the current stream) are appended."""
        v, f = [vx, vy, vz], (None if fx is None else [fx, fy, fz])
        for t in range(nsteps):
            for o in range(ord, 0, -1):
                pr = not (t == 0 and o == ord)
                self.front(v, o == ord, pr)
                if self.nranks == 1:
                    self.xpass(pr)
                else:
                    for d in (0, 1):
                        self.pack(d, pr)
                        if exchange_events is not None:
                            e0 = torch.cuda.Event(enable_timing=True)
                            e0.record()
                        all_to_all(self.recv, self.send, self.counts[d, pr][1], self.counts[d, pr][0], group)
                        if exchange_events is not None:
                            e1 = torch.cuda.Event(enable_timing=True)
                            e1.record()
                            exchange_events.append((e0, e1))
                        self.unpack(d, pr)
                        if d == 0:
                            self.xpass(pr)
                self.back(o, dt, nu, v, f, pr)


def _local_exchange(slabs, direction: int, prune: bool):
    """The all-to-all among ranks held by one process: device copies from
    every peer's send chunk for r into r's receive chunk from that peer."""
    n = len(slabs)
    for r, dst in enumerate(slabs):
        roff = 0
        rc = dst.counts[direction, prune][1]
        for p, src in enumerate(slabs):
            sc = src.counts[direction, prune][0]
            soff = sum(sc[:r])
            assert sc[r] == rc[p]
            dst.recv[roff:roff + rc[p]].copy_(src.send[soff:soff + sc[r]])
            roff += rc[p]
    return n


def run_local(slabs, nsteps: int, ord: int, dt: float, nu: float, vs, fs=None):
    """RK steps of a decomposed run whose ranks this process holds (slabs
    in rank order, vs[r] / fs[r] rank r's kx-slabs of v and f): the same
    library calls as Slab.run, phase by phase over the ranks, with the
    all-to-alls done by device copies on the current stream."""
    for t in range(nsteps):
        for o in range(ord, 0, -1):
            pr = not (t == 0 and o == ord)
            for s, v in zip(slabs, vs):
                s.front(v, o == ord, pr)
            if len(slabs) == 1:
                slabs[0].xpass(pr)
            for d in (0, 1) if len(slabs) > 1 else ():
                for s in slabs:
                    s.pack(d, pr)
                _local_exchange(slabs, d, pr)
                for s in slabs:
                    s.unpack(d, pr)
                if d == 0:
                    for s in slabs:
                        s.xpass(pr)
            for r, (s, v) in enumerate(zip(slabs, vs)):
                s.back(o, dt, nu, v, None if fs is None else fs[r], pr)
