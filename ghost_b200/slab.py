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

By default (Slab(overlap=True)) the exchanges are split into field groups
(substep(), GROUPS_OVERLAP): the all-to-all of v's three fields runs while
curl v is transformed along y, and each product field's all-to-all back
runs while the previous field is transformed along y; the collectives are
asynchronous, each on its own buffer slot, and a rank's own block moves
field to field (ghost_slab_exchange_self) instead of through the buffers.
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


def exchange_counts(nxhl, nzl, ny: int, rank: int, direction: int, nf: int, self_direct: bool = False):
    """Complex values sent to and received from every peer by `rank` in one
    all-to-all of nf fields.  Direction 0 (kx-slab -> z-slab): the chunk
    for peer p is nf blocks of my kx rows x ny x p's z planes; the chunk
    from p is nf blocks of p's rows x ny x my planes.  Direction 1 is the
    reverse.  For a pruned exchange nxhl is the ranks' live rows.  With
    self_direct the rank's own chunk is empty (it moves field to field)."""
    n = len(nxhl)
    mine = [nf * nxhl[rank] * ny * nzl[p] for p in range(n)]
    theirs = [nf * nxhl[p] * ny * nzl[rank] for p in range(n)]
    if self_direct:
        mine[rank] = theirs[rank] = 0
    return (mine, theirs) if direction == 0 else (theirs, mine)


# Field groups of the two exchanges of a substep.  Plain: one all-to-all of
# the six front fields, one of the three x-pass products.  Overlapped: the
# front's fields go in two groups (v, then curl v), so that the first
# group's all-to-all runs while the second group is transformed along y;
# the products go one field at a time, so that field q's Y forward runs
# while the later fields are still in flight.
GROUPS_PLAIN = (((0, 1, 2, 3, 4, 5),), ((0, 1, 2),))
GROUPS_OVERLAP = (((0, 1, 2), (3, 4, 5)), ((0,), (1,), (2,)))


def substep(ops, o, dt, nu, v, f, copy, prune, groups, self_direct):
    """One HD substep of a slab-decomposed run (include/hd_rkstep2.f90) as
    a schedule of phases over field groups.  ops provides the phases for one
    rank (Slab) or for all ranks in lockstep (run_local):
      front_z(v, copy, prune); ypass(sign, idx, prune);
      pack(d, idx, prune, g); exchange(d, g, nf, prune) -> handle;
      wait(handle); unpack(d, idx, prune, g); exchange_self(d, idx, prune);
      xpass(prune); back_z(o, dt, nu, v, f, prune).
    Group g of direction d has its own buffer slot, so that no pack or
    unpack touches the buffers of an all-to-all in flight.  The results do
    not depend on the grouping (a line's arithmetic is the same), nor on
    self_direct."""
    g0, g1 = groups
    ops.front_z(v, copy, prune)
    hs = []
    for g, idx in enumerate(g0):
        ops.ypass(+1, idx, prune)
        ops.pack(0, idx, prune, g)
        hs.append(ops.exchange(0, g, len(idx), prune))
    if self_direct:
        ops.exchange_self(0, tuple(q for idx in g0 for q in idx), prune)
    for g, idx in enumerate(g0):
        ops.wait(hs[g])
        ops.unpack(0, idx, prune, g)
    ops.xpass(prune)
    hs = []
    for g, idx in enumerate(g1):
        ops.pack(1, idx, prune, g)
        hs.append(ops.exchange(1, g, len(idx), prune))
    if self_direct:
        ops.exchange_self(1, tuple(q for idx in g1 for q in idx), prune)
    for g, idx in enumerate(g1):
        ops.wait(hs[g])
        ops.unpack(1, idx, prune, g)
        ops.ypass(-1, idx, prune)
    ops.back_z(o, dt, nu, v, f, prune)


def all_to_all(recv, send, recv_counts, send_counts, group=None, async_op=False):
    """One all-to-all of complex buffers (peer-major chunks of the given
    counts) over torch.distributed; the buffers travel as their real
    and imaginary parts.  async_op: returns the work handle, whose wait()
    orders the caller's stream after the exchange."""
    import torch.distributed as dist
    r = torch.view_as_real(recv[:sum(recv_counts)]).reshape(-1)
    s = torch.view_as_real(send[:sum(send_counts)]).reshape(-1)
    return dist.all_to_all_single(r, s, [2 * c for c in recv_counts], [2 * c for c in send_counts], group=group,
                                  async_op=async_op)


class Slab:
    """One rank's share of a slab-decomposed HD run: the library's slab
    context and the work arrays of the substep.

    overlap (default): the exchanges go in field groups (GROUPS_OVERLAP),
    each all-to-all asynchronous on its own buffer slot and overlapped with
    the Y passes of the other groups, and the rank's own block moves field
    to field (ghost_slab_exchange_self) instead of through the buffers.
    overlap=False: one synchronous all-to-all per direction carrying every
    block, the own block included."""

    def __init__(self, nx: int, ny: int | None = None, nz: int | None = None, Lx: float = 1.0, Ly: float = 1.0,
                 Lz: float = 1.0, arbsize: bool = False, precision: str = "fp64", rank: int = 0, nranks: int = 1,
                 stream=None, overlap: bool = True):
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
        # buffers for either mode (the plain one's hold the most)
        nsend = nrecv = 0
        for ov in (False, True):
            self.set_overlap(ov, _sizes_only=True)
            nsend, nrecv = max(nsend, self._nsend), max(nrecv, self._nrecv)
        self.send = torch.empty(max(nsend, 1), dtype=dt, device=dev)
        self.recv = torch.empty(max(nrecv, 1), dtype=dt, device=dev)
        self.group = None
        self.exchange_events = None
        self.set_overlap(overlap)

    def set_overlap(self, on: bool, _sizes_only: bool = False):
        """Switch between the overlapped schedule (field groups, asynchronous
        all-to-alls, own block field to field) and the plain one; one rank
        always runs the plain one (it has no exchange)."""
        self.overlap = bool(on) and self.nranks > 1
        self.self_direct = self.overlap
        self.groups = GROUPS_OVERLAP if self.overlap else GROUPS_PLAIN
        # buffer slots: group g of direction d at send/recv offsets soff/roff[d, g]
        # (the two directions never have exchanges in flight together, so they share the buffers)
        self.soff, self.roff = {}, {}
        self._nsend = self._nrecv = 0
        for d in (0, 1):
            so = ro = 0
            for g, idx in enumerate(self.groups[d]):
                sc, rc = self.counts(d, len(idx), False)
                self.soff[d, g], self.roff[d, g] = so, ro
                so += sum(sc)
                ro += sum(rc)
            self._nsend, self._nrecv = max(self._nsend, so), max(self._nrecv, ro)
        if not _sizes_only:
            check(self.lib.ghost_slab_set_self_direct(self.h, int(self.self_direct)), "ghost_slab_set_self_direct")

    def counts(self, d: int, nf: int, prune: bool):
        """(send counts, receive counts) of an exchange of nf fields in direction d."""
        return exchange_counts(live_rows(self.ista, self.nxhl, self.rows if prune else None), self.nzl, self.ny,
                               self.rank, d, nf, self.self_direct)

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

    def front_z(self, v, copy: bool, prune: bool = False):
        check(self.lib.ghost_slab_hd_front_z(self.h, self._pp(self._fields(v)), self._pp(self.C), int(copy),
                                             int(prune), self._pp(self.w)), "ghost_slab_hd_front_z")

    def ypass(self, sign: int, idx, prune: bool = False):
        check(self.lib.ghost_slab_ypass(self.h, sign, len(idx), int(prune), self._pp([self.w[q] for q in idx])),
              "ghost_slab_ypass")

    def _slot(self, buf, off, d, g):
        return ctypes.c_void_p(buf[off[d, g]:].data_ptr())

    def pack(self, direction: int, idx=None, prune: bool = False, g: int = 0):
        if idx is None:
            idx = self.groups[direction][0]
        fields = [(self.w if direction == 0 else self.z)[q] for q in idx]
        check(self.lib.ghost_slab_pack(self.h, direction, len(fields), int(prune), self._pp(fields),
                                       self._slot(self.send, self.soff, direction, g)), "ghost_slab_pack")

    def unpack(self, direction: int, idx=None, prune: bool = False, g: int = 0):
        if idx is None:
            idx = self.groups[direction][0]
        fields = [(self.z if direction == 0 else self.w)[q] for q in idx]
        check(self.lib.ghost_slab_unpack(self.h, direction, len(fields), int(prune),
                                         self._slot(self.recv, self.roff, direction, g), self._pp(fields)),
              "ghost_slab_unpack")

    def exchange(self, direction: int, g: int, nf: int, prune: bool = False):
        """The all-to-all of group g: asynchronous with overlap (returns the
        work handle), else synchronous (events around it when requested)."""
        sc, rc = self.counts(direction, nf, prune)
        send = self.send[self.soff[direction, g]:]
        recv = self.recv[self.roff[direction, g]:]
        if self.overlap:
            return all_to_all(recv, send, rc, sc, self.group, async_op=True)
        if self.exchange_events is not None:
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record()
        all_to_all(recv, send, rc, sc, self.group)
        if self.exchange_events is not None:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record()
            self.exchange_events.append((e0, e1))
        return None

    @staticmethod
    def wait(handle):
        if handle is not None:
            handle.wait()

    def exchange_self(self, direction: int, idx, prune: bool = False):
        src, dst = (self.w, self.z) if direction == 0 else (self.z, self.w)
        check(self.lib.ghost_slab_exchange_self(self.h, direction, len(idx), int(prune), self._pp([src[q] for q in idx]),
                                                self._pp([dst[q] for q in idx])), "ghost_slab_exchange_self")

    def xpass(self, prune: bool = False):
        # one rank: the kx-slab is the whole field and the z-slab layout is the same, so the x pass
        # runs on the front's output in place and no exchange is needed
        z = self.w if self.nranks == 1 else self.z
        check(self.lib.ghost_slab_hd_xpass(self.h, int(prune), self._pp(z), self._pp(z[:3])), "ghost_slab_hd_xpass")

    def back(self, o: int, dt: float, nu: float, v, f=None, prune: bool = False):
        fp = self._pp(self._fields(f)) if f is not None else None
        check(self.lib.ghost_slab_hd_back(self.h, o, dt, nu, int(prune), self._pp(self.w[:3]),
                                          self._pp(self._fields(v)), self._pp(self.C), fp), "ghost_slab_hd_back")

    def back_z(self, o: int, dt: float, nu: float, v, f=None, prune: bool = False):
        fp = self._pp(self._fields(f)) if f is not None else None
        check(self.lib.ghost_slab_hd_back_z(self.h, o, dt, nu, int(prune), self._pp(self.w[:3]),
                                            self._pp(self._fields(v)), self._pp(self.C), fp), "ghost_slab_hd_back_z")

    # -- runs -----------------------------------------------------------
    def run(self, nsteps: int, ord: int, dt: float, nu: float, vx, vy, vz, fx=None, fy=None, fz=None, group=None,
            exchange_events=None):
        """nsteps RK steps of order ord (GHOST's RK loop, main3D.fpp:3195-3231)
        of this rank's kx-slab of v, the transposes as NCCL all-to-alls.
        Every substep after the first is zero-pruned, as in ghost_hd_run.
        exchange_events (synchronous exchanges only, overlap=False): a list to
        which CUDA event pairs bracketing each all-to-all (on the current
        stream) are appended."""
        if exchange_events is not None and self.overlap:
            raise ValueError("exchange_events times synchronous exchanges: construct the Slab with overlap=False")
        v, f = [vx, vy, vz], (None if fx is None else [fx, fy, fz])
        self.group, self.exchange_events = group, exchange_events
        try:
            for t in range(nsteps):
                for o in range(ord, 0, -1):
                    pr = not (t == 0 and o == ord)
                    if self.nranks == 1:
                        self.front(v, o == ord, pr)
                        self.xpass(pr)
                        self.back(o, dt, nu, v, f, pr)
                    else:
                        substep(self, o, dt, nu, v, f, o == ord, pr, self.groups, self.self_direct)
        finally:
            self.group, self.exchange_events = None, None


class _Lockstep:
    """The phases of substep() applied to every rank that one process holds,
    rank after rank; an exchange is the device copies from every peer's send
    slot for r into r's receive slot from that peer, once every rank has
    packed."""

    def __init__(self, slabs):
        self.slabs = slabs

    def front_z(self, vs, copy, prune):
        for s, v in zip(self.slabs, vs):
            s.front_z(v, copy, prune)

    def ypass(self, sign, idx, prune):
        for s in self.slabs:
            s.ypass(sign, idx, prune)

    def pack(self, d, idx, prune, g):
        for s in self.slabs:
            s.pack(d, idx, prune, g)

    def exchange(self, d, g, nf, prune):
        for r, dst in enumerate(self.slabs):
            rc = dst.counts(d, nf, prune)[1]
            roff = dst.roff[d, g]
            for p, src in enumerate(self.slabs):
                sc = src.counts(d, nf, prune)[0]
                soff = src.soff[d, g] + sum(sc[:r])
                assert sc[r] == rc[p]
                if rc[p]:
                    dst.recv[roff:roff + rc[p]].copy_(src.send[soff:soff + sc[r]])
                roff += rc[p]
        return None

    @staticmethod
    def wait(handle):
        pass

    def unpack(self, d, idx, prune, g):
        for s in self.slabs:
            s.unpack(d, idx, prune, g)

    def exchange_self(self, d, idx, prune):
        for s in self.slabs:
            s.exchange_self(d, idx, prune)

    def xpass(self, prune):
        for s in self.slabs:
            s.xpass(prune)

    def back_z(self, o, dt, nu, vs, fs, prune):
        for r, (s, v) in enumerate(zip(self.slabs, vs)):
            s.back_z(o, dt, nu, v, None if fs is None else fs[r], prune)


def run_local(slabs, nsteps: int, ord: int, dt: float, nu: float, vs, fs=None):
    """RK steps of a decomposed run whose ranks this process holds (slabs
    in rank order, vs[r] / fs[r] rank r's kx-slabs of v and f): the same
    schedule and library calls as Slab.run (the slabs' overlap setting
    picks the field groups), phase by phase over the ranks, with the
    all-to-alls done by device copies on the current stream."""
    if len(slabs) == 1:
        s = slabs[0]
        return s.run(nsteps, ord, dt, nu, *vs[0], *(fs[0] if fs is not None else (None, None, None)))
    ops = _Lockstep(slabs)
    groups, direct = slabs[0].groups, slabs[0].self_direct
    if any(s.groups != groups or s.self_direct != direct for s in slabs):
        raise ValueError("the ranks of a run need the same overlap setting")
    for t in range(nsteps):
        for o in range(ord, 0, -1):
            pr = not (t == 0 and o == ord)
            substep(ops, o, dt, nu, vs, fs, o == ord, pr, groups, direct)
