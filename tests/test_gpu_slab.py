"""The slab-decomposed HD run on one GPU: the ranks of a decomposed run
held by one process (ghost_b200.slab.run_local: the library's slab passes,
packing and unpacking, with the all-to-alls done by device copies), against
the undivided run of ghost_hd_run on the same fields.  Uneven kx slabs
(33 rows over 2 or 4 ranks) included.  Both schedules: the overlapped one
(field groups, own block copied field to field) and the plain one, which
give the same bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fields(g, seed):
    v = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(seed, 1.0, g.nx / 3.0, 1, 1.0, *v)
    return v


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("prec,P,shape", [("fp64", 1, (64, 64, 64)), ("fp64", 2, (64, 64, 64)),
                                          ("fp64", 4, (64, 64, 64)), ("fp32", 2, (64, 64, 64)),
                                          ("fp64", 4, (64, 32, 128))])
def test_slab_run_matches_undivided_run(prec, P, shape, overlap):
    import torch

    from ghost_b200 import Ghost
    from ghost_b200.slab import Slab, run_local
    nx, ny, nz = shape
    arb = shape != (nx, nx, nx)
    kw = dict(Lx=1.0, Ly=2.0, Lz=0.5, arbsize=True) if arb else {}
    g = Ghost(nx, ny, nz, precision=prec, **kw)
    v0, f = _fields(g, 1000), _fields(g, 77)
    ref = [x.clone() for x in v0]
    g.hd_run(2, 4, 1e-3, 2e-3, *ref, *f)
    slabs = [Slab(nx, ny, nz, precision=prec, rank=r, nranks=P, overlap=overlap, **kw) for r in range(P)]
    vs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in v0] for r, s in enumerate(slabs)]
    fs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in f] for r, s in enumerate(slabs)]
    for _ in range(2):  # two calls in a row: the work arrays carry nothing over
        vv = [[x.clone() for x in v] for v in vs]
        run_local(slabs, 2, 4, 1e-3, 2e-3, vv, fs)
        torch.cuda.synchronize()
        got = [torch.cat([vv[r][c] for r in range(P)], dim=0) for c in range(3)]
        for c in range(3):
            a, b = got[c].cpu().numpy(), ref[c].cpu().numpy()
            err = np.abs(a - b).max() / np.abs(b).max()
            assert err <= (1e-12 if prec == "fp64" else 1e-5), (c, err)
    for s in slabs:
        s.close()


def test_slab_phases_reject_host_and_misshaped_arrays():
    from ghost_b200.slab import Slab
    s = Slab(64, precision="fp64", rank=1, nranks=2)
    with pytest.raises(ValueError):
        s.front([t[:-1] for t in s.C], True)
    s.close()


def test_slab_run_without_forcing_and_null_forcing_pointers():
    """No forcing: f NULL (Python None) and f an array of three null
    pointers (a Fortran caller's C_NULL_PTRs) both mean none, against the
    undivided run without forcing.  FP32, 4 ranks (one without live rows)."""
    import ctypes

    import torch

    from ghost_b200 import Ghost
    from ghost_b200.slab import Slab, run_local
    g = Ghost(64, precision="fp32")
    v0 = _fields(g, 1000)
    ref = [x.clone() for x in v0]
    g.hd_run(1, 2, 1e-3, 2e-3, *ref)
    P = 4
    slabs = [Slab(64, precision="fp32", rank=r, nranks=P) for r in range(P)]
    assert slabs[0].rows == 22 and slabs[3].ista[3] >= 22   # the last rank holds no live kx row
    vs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in v0] for r, s in enumerate(slabs)]
    run_local(slabs, 1, 2, 1e-3, 2e-3, vs, None)
    torch.cuda.synchronize()
    for c in range(3):
        got = torch.cat([vs[r][c] for r in range(P)], dim=0)
        err = ((got - ref[c]).abs().max() / ref[c].abs().max()).item()
        assert err <= 1e-5, (c, err)
    # one substep's back phase with three null forcing pointers equals it with f = NULL
    s = Slab(64, precision="fp64", rank=0, nranks=1)
    g64 = Ghost(64, precision="fp64")
    v = _fields(g64, 5)
    outs = []
    for nullarr in (False, True):
        w = [x.clone() for x in v]
        s.front(w, True)
        s.xpass()
        f = (ctypes.c_void_p * 3)(None, None, None) if nullarr else None
        st = s.lib.ghost_slab_hd_back(s.h, 1, 1e-3, 2e-3, 0, s._pp(s.w[:3]), s._pp(w), s._pp(s.C), f)
        assert st == 0, s.lib.ghost_last_error_string()
        torch.cuda.synchronize()
        outs.append([x.clone() for x in w])
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    for t in slabs + [s]:
        t.close()


@pytest.mark.parametrize("prec,P", [("fp32", 2), ("fp64", 2), ("fp32", 4), ("fp64", 4)])
def test_overlapped_schedule_is_the_plain_one_bit_for_bit(prec, P):
    """Field groups, asynchronous slots and the own block copied field to
    field change no bit of the run (uneven kx slabs: 33 rows over 2 or 4
    ranks; with 4 ranks one holds no live row)."""
    import torch

    from ghost_b200 import Ghost
    from ghost_b200.slab import Slab, run_local
    nz = 64
    g = Ghost(64, 64, nz, precision=prec)
    v0, f = _fields(g, 31), _fields(g, 32)
    out = {}
    for overlap in (True, False):
        slabs = [Slab(64, 64, nz, precision=prec, rank=r, nranks=P, overlap=overlap) for r in range(P)]
        assert all(s.overlap == overlap and s.self_direct == overlap for s in slabs)
        vs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in v0] for r, s in enumerate(slabs)]
        fs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in f] for r, s in enumerate(slabs)]
        run_local(slabs, 2, 3, 1e-3, 2e-3, vs, fs)
        torch.cuda.synchronize()
        out[overlap] = [torch.cat([vs[r][c] for r in range(P)], dim=0) for c in range(3)]
        for s in slabs:
            s.close()
    for a, b in zip(out[True], out[False]):
        assert torch.equal(a, b)
    # switching a slab's mode at run time gives the same bits again
    slabs = [Slab(64, 64, nz, precision=prec, rank=r, nranks=P, overlap=False) for r in range(P)]
    for s in slabs:
        s.set_overlap(True)
    vs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in v0] for r, s in enumerate(slabs)]
    fs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in f] for r, s in enumerate(slabs)]
    run_local(slabs, 2, 3, 1e-3, 2e-3, vs, fs)
    torch.cuda.synchronize()
    for c in range(3):
        assert torch.equal(torch.cat([vs[r][c] for r in range(P)], dim=0), out[False][c])
    for s in slabs:
        s.close()
