"""Slab decomposition host logic (no GPU): GHOST's range() through the
library, the exchange counts, and the all-to-all of ghost_b200.slab over a
two-rank gloo group with blocks packed in the documented peer-major layout
(the device packing is checked on the GPU in test_gpu_slab.py)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _range_ref(n1, n2, nprocs, irank):
    # fftp-3/fftp.f90 SUBROUTINE range, as written there
    iwork1 = (n2 - n1 + 1) // nprocs
    iwork2 = (n2 - n1 + 1) % nprocs
    ista = irank * iwork1 + n1 + min(irank, iwork2)
    iend = ista + iwork1 - 1
    if iwork2 > irank:
        iend += 1
    return ista, iend


@pytest.mark.parametrize("n", [16, 33, 257, 512, 513])
@pytest.mark.parametrize("p", [1, 2, 3, 4, 7, 8])
def test_range_is_ghosts_and_tiles_the_axis(n, p):
    from ghost_b200.slab import slab_range
    got = [slab_range(1, n, p, r) for r in range(p)]
    assert got == [_range_ref(1, n, p, r) for r in range(p)]
    assert got[0][0] == 1 and got[-1][1] == n
    assert all(got[r][1] + 1 == got[r + 1][0] for r in range(p - 1))
    sizes = [b - a + 1 for a, b in got]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_slab_create_rejects_what_it_cannot_split():
    from ghost_b200 import _lib
    import ctypes
    lib = _lib.load()
    h = ctypes.c_void_p()
    # 64 planes over 3 ranks: 22/21/21, not multiples of 8 (checked before any device is touched)
    assert lib.ghost_slab_create(64, 64, 64, 1., 1., 1., 0, 8, 0, 3, ctypes.byref(h)) == 2
    assert lib.ghost_slab_create(64, 64, 64, 1., 1., 1., 0, 8, 3, 3, ctypes.byref(h)) == 1


@pytest.mark.parametrize("nx,nz,p", [(64, 64, 2), (64, 64, 4), (512, 512, 8), (32, 128, 4)])
def test_exchange_counts_match_between_peers(nx, nz, p):
    from ghost_b200.slab import exchange_counts, slab_layout
    ista, nxhl, ksta, nzl = slab_layout(nx, nz, p)
    assert sum(nxhl) == nx // 2 + 1 and sum(nzl) == nz
    ny = 16
    for d, nf in ((0, 6), (1, 3)):
        c = [exchange_counts(nxhl, nzl, ny, r, d, nf) for r in range(p)]
        for r in range(p):
            for q in range(p):
                assert c[r][0][q] == c[q][1][r]     # what r sends q is what q expects from r
        # every value of the nf fields moves exactly once
        assert sum(sum(x[0]) for x in c) == nf * (nx // 2 + 1) * ny * nz
    # pruned: only the rows below the live count, each exactly once
    from ghost_b200.slab import live_rows
    rows = (nx // 3) + 1
    lr = live_rows(ista, nxhl, rows)
    assert sum(lr) == rows and all(0 <= a <= b for a, b in zip(lr, nxhl))
    assert all(lr[r] == nxhl[r] for r in range(p) if ista[r] + nxhl[r] <= rows)
    c = [exchange_counts(lr, nzl, ny, r, 0, 6) for r in range(p)]
    assert sum(sum(x[0]) for x in c) == 6 * rows * ny * nz


def test_slab_roofline_counts_the_busiest_ranks_link_bytes():
    """The roofline of the slab line: 64^3 over 2 ranks holds kx rows 17/16,
    of which 17/5 are live (kx <= 21).  Rank 0 sends v and curl v of its 17
    live rows for rank 1's 32 planes and the three products of rank 1's 5
    live rows back: 6*17*64*32 + 3*5*64*32 complex values, the largest load
    of either rank in either direction.  The HBM share is the undivided
    run's pruned bytes over the ranks."""
    from ghost_b200.roofline import pass_bytes, slab_exchange_bytes, slab_roofline
    assert slab_exchange_bytes(64, 2) == (6 * 17 * 64 * 32 + 3 * 5 * 64 * 32) * 8
    assert slab_exchange_bytes(64, 2, elem_bytes=16) == 2 * slab_exchange_bytes(64, 2)
    r = slab_roofline(64, 2, ms_per_step=2.0, xch_ms_per_substep=0.5)
    step_bytes = 4 * sum(pass_bytes(64, 4).values()) / 2
    assert r["bytes_per_rank_per_step"] == pytest.approx(step_bytes)
    assert r["achieved"] == pytest.approx(step_bytes / 2e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert r["exchange"]["achieved"] == pytest.approx(slab_exchange_bytes(64, 2) / 0.5e-3 / 1e9)
    assert r["exchange"]["frac"] == pytest.approx(r["exchange"]["achieved"] / 770.0)
    # one rank exchanges nothing
    assert slab_exchange_bytes(64, 1) == 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pack(fields_k, direction, me, ista, nxhl, ksta, nzl):
    # the documented peer-major layout, restated with numpy
    out = []
    for p in range(len(nxhl)):
        for f in fields_k:
            if direction == 0:
                out.append(f[:, :, ksta[p]:ksta[p] + nzl[p]].ravel())
            else:
                out.append(f[ista[p]:ista[p] + nxhl[p]].ravel())
    return np.concatenate(out)


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from ghost_b200.slab import all_to_all, exchange_counts, slab_layout
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    nx, ny, nz, nf = 32, 4, 32, 2
    ista, nxhl, ksta, nzl = slab_layout(nx, nz, ws)
    rng = np.random.default_rng(5)
    glob = [rng.standard_normal((nx // 2 + 1, ny, nz)) + 1j * rng.standard_normal((nx // 2 + 1, ny, nz))
            for _ in range(nf)]
    mine_k = [g[ista[rank]:ista[rank] + nxhl[rank]] for g in glob]
    # kx-slab -> z-slab
    sc, rc = exchange_counts(nxhl, nzl, ny, rank, 0, nf)
    send = torch.from_numpy(_pack(mine_k, 0, rank, ista, nxhl, ksta, nzl))
    recv = torch.zeros(sum(rc), dtype=torch.complex128)
    all_to_all(recv, send, rc, sc)
    r = recv.numpy()
    z = [np.zeros((nx // 2 + 1, ny, nzl[rank]), complex) for _ in range(nf)]
    off = 0
    for p in range(ws):
        for f in range(nf):
            n = nxhl[p] * ny * nzl[rank]
            z[f][ista[p]:ista[p] + nxhl[p]] = r[off:off + n].reshape(nxhl[p], ny, nzl[rank])
            off += n
    ok0 = all(np.array_equal(z[f], glob[f][:, :, ksta[rank]:ksta[rank] + nzl[rank]]) for f in range(nf))
    # and back
    sc, rc = exchange_counts(nxhl, nzl, ny, rank, 1, nf)
    send = torch.from_numpy(_pack(z, 1, rank, ista, nxhl, ksta, nzl))
    recv = torch.zeros(sum(rc), dtype=torch.complex128)
    all_to_all(recv, send, rc, sc)
    r = recv.numpy()
    k = [np.zeros_like(m) for m in mine_k]
    off = 0
    for p in range(ws):
        for f in range(nf):
            n = nxhl[rank] * ny * nzl[p]
            k[f][:, :, ksta[p]:ksta[p] + nzl[p]] = r[off:off + n].reshape(nxhl[rank], ny, nzl[p])
            off += n
    ok1 = all(np.array_equal(k[f], mine_k[f]) for f in range(nf))
    with open(os.path.join(out, f"r{rank}"), "w") as fh:
        fh.write(f"{int(ok0)}{int(ok1)}")
    dist.destroy_process_group()


def test_transposes_over_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert [open(tmp_path / f"r{r}").read() for r in range(2)] == ["11", "11"]


class _FakeOps:
    """The phases of ghost_b200.slab.substep for one gloo rank on CPU
    tensors: the documented pack/unpack layouts and the own-block copy
    restated with torch, and the passes replaced by elementwise maps, a
    different one per phase and field, so that a misplaced block, a wrong
    group, a reused buffer slot or a missing wait changes the result."""

    def __init__(self, nx, ny, nz, ws, rank, groups, self_direct):
        import torch

        from ghost_b200.slab import slab_layout
        self.ny, self.ws, self.rank, self.direct = ny, ws, rank, self_direct
        self.ista, self.nxhl, self.ksta, self.nzl = slab_layout(nx, nz, ws)
        kshape, zshape = (self.nxhl[rank], ny, nz), (nx // 2 + 1, ny, self.nzl[rank])
        self.w = [torch.zeros(kshape, dtype=torch.complex128) for _ in range(6)]
        self.z = [torch.zeros(zshape, dtype=torch.complex128) for _ in range(6)]
        self.C = [torch.zeros(kshape, dtype=torch.complex128) for _ in range(3)]
        self.slots = {}

    def front_z(self, v, copy, prune):
        for a in range(3):
            self.w[a] = v[a].clone()
            self.w[3 + a] = v[a] * (0.5 + 0.25j) + (a + 1)
            if copy:
                self.C[a] = v[a].clone()

    def ypass(self, sign, idx, prune):
        for q in idx:
            self.w[q] = self.w[q] * (1.25 if sign > 0 else 0.75 - 0.1j) + 0.125 * (q + 1) * sign

    def _peers(self):
        return [p for p in range(self.ws) if not (self.direct and p == self.rank)]

    def pack(self, d, idx, prune, g):
        import torch
        me, parts = self.rank, []
        for p in self._peers():
            for q in idx:
                if d == 0:
                    parts.append(self.w[q][:, :, self.ksta[p]:self.ksta[p] + self.nzl[p]].reshape(-1))
                else:
                    parts.append(self.z[q][self.ista[p]:self.ista[p] + self.nxhl[p]].reshape(-1))
        self.slots[d, g] = [torch.cat(parts) if parts else torch.zeros(0, dtype=torch.complex128), None, idx]

    def exchange(self, d, g, nf, prune):
        import torch

        from ghost_b200.slab import all_to_all, exchange_counts
        sc, rc = exchange_counts(self.nxhl, self.nzl, self.ny, self.rank, d, nf, self.direct)
        slot = self.slots[d, g]
        slot[1] = torch.zeros(sum(rc), dtype=torch.complex128)
        return all_to_all(slot[1], slot[0], rc, sc, async_op=True)

    @staticmethod
    def wait(h):
        if h is not None:
            h.wait()

    def unpack(self, d, idx, prune, g):
        me, r, off = self.rank, self.slots[d, g][1], 0
        for p in self._peers():
            for q in idx:
                if d == 0:
                    n = self.nxhl[p] * self.ny * self.nzl[me]
                    self.z[q][self.ista[p]:self.ista[p] + self.nxhl[p]] = r[off:off + n].reshape(
                        self.nxhl[p], self.ny, self.nzl[me])
                else:
                    n = self.nxhl[me] * self.ny * self.nzl[p]
                    self.w[q][:, :, self.ksta[p]:self.ksta[p] + self.nzl[p]] = r[off:off + n].reshape(
                        self.nxhl[me], self.ny, self.nzl[p])
                off += n

    def exchange_self(self, d, idx, prune):
        me = self.rank
        rows, planes = slice(self.ista[me], self.ista[me] + self.nxhl[me]), slice(self.ksta[me],
                                                                                self.ksta[me] + self.nzl[me])
        for q in idx:
            if d == 0:
                self.z[q][rows] = self.w[q][:, :, planes]
            else:
                self.w[q][:, :, planes] = self.z[q][rows]

    def xpass(self, prune):
        for a in range(3):
            self.z[a] = self.z[a] * self.z[a + 3] + 0.5

    def back_z(self, o, dt, nu, v, f, prune):
        for a in range(3):
            v[a].copy_(self.C[a] + dt * (self.w[a] - nu * v[a] + (f[a] if f is not None else 0)) / o)


def _fake_undivided(glob_v, glob_f, nsteps, ord, dt, nu):
    """The same fake phases on the whole field, with no exchange."""
    out = [x.clone() for x in glob_v]
    for t in range(nsteps):
        C = [x.clone() for x in out]
        for o in range(ord, 0, -1):
            w = [x.clone() for x in out] + [x * (0.5 + 0.25j) + (a + 1) for a, x in enumerate(out)]
            w = [x * 1.25 + 0.125 * (q + 1) for q, x in enumerate(w)]
            w = [w[a] * w[a + 3] + 0.5 for a in range(3)]
            w = [x * (0.75 - 0.1j) - 0.125 * (q + 1) for q, x in enumerate(w)]
            out = [C[a] + dt * (w[a] - nu * out[a] + glob_f[a]) / o for a in range(3)]
    return out


def _schedule_worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from ghost_b200.slab import GROUPS_OVERLAP, GROUPS_PLAIN, substep
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    nx, ny, nz = 32, 4, 24
    rng = np.random.default_rng(11)
    shape = (nx // 2 + 1, ny, nz)
    gv = [torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) for _ in range(3)]
    gf = [torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) for _ in range(3)]
    ref = _fake_undivided(gv, gf, 2, 3, 1e-2, 0.3)
    res = {}
    for name, groups, direct in (("plain", GROUPS_PLAIN, False), ("overlap", GROUPS_OVERLAP, True)):
        ops = _FakeOps(nx, ny, nz, ws, rank, groups, direct)
        lo, n = ops.ista[rank], ops.nxhl[rank]
        v = [x[lo:lo + n].clone() for x in gv]
        f = [x[lo:lo + n].clone() for x in gf]
        for t in range(2):
            for o in range(3, 0, -1):
                substep(ops, o, 1e-2, 0.3, v, f, o == 3, False, groups, direct)
        res[name] = v
        ok = all(torch.allclose(v[a], ref[a][lo:lo + n], rtol=1e-12, atol=1e-12) for a in range(3))
        res[name + "_ok"] = ok
    same = all(torch.equal(a, b) for a, b in zip(res["plain"], res["overlap"]))
    with open(os.path.join(out, f"s{rank}"), "w") as fh:
        fh.write(f"{int(res['plain_ok'])}{int(res['overlap_ok'])}{int(same)}")
    dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_overlapped_schedule_over_gloo(tmp_path, ws):
    """substep() over real gloo ranks with asynchronous all-to-alls: the
    overlapped schedule (field groups, own block field to field) and the
    plain one both give the undivided result, and the same bits."""
    import torch.multiprocessing as mp
    mp.start_processes(_schedule_worker, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    assert [open(tmp_path / f"s{r}").read() for r in range(ws)] == ["111"] * ws
