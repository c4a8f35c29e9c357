"""Throughput of the slab-decomposed HD run (GHOST's kx-slab / z-slab layout).

    python -m ghost_b200.slab_bench --n 512 --ranks 2        # P ranks held by one process on one GPU
    torchrun --nproc-per-node N -m ghost_b200.slab_bench --n 1024   # one rank per GPU, NCCL all-to-alls

With one process the ranks' passes run one after the other on one GPU and
the all-to-alls are device copies (ghost_b200.slab.run_local), so the rate
is that of one GPU doing every rank's work: a check of the decomposition's
overhead (the packing, unpacking and copies) against the undivided run, not
of scaling.  Under torchrun every rank times its own run with CUDA events
after a barrier and the time is the maximum over ranks.  Forced HD, RK4,
seeded solenoidal fields, no zero-pruning.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--ranks", type=int, default=1, help="ranks held by this process (single-process mode)")
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    a = ap.parse_args(argv)

    import torch

    from ghost_b200 import Ghost
    from ghost_b200.slab import Slab, run_local

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    n, dt, nu = a.n, 5e-4, 1e-3
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    g = Ghost(n, precision=a.precision)
    v = [g.czeros() for _ in range(3)]
    f = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, n / 3.0, 1, 1.0, *v)
    g.init_random_solenoidal(77, 1.0, 3.0, 1, 1.0, *f)
    if world > 1:
        s = Slab(n, precision=a.precision, rank=rank, nranks=world)
        lo, cnt = s.ista[rank], s.nxhl[rank]
        vs = [x[lo:lo + cnt].clone() for x in v]
        fs = [x[lo:lo + cnt].clone() for x in f]
        del v, f, g
        step = lambda k: s.run(k, 4, dt, nu, *vs, *fs)
        ranks = world
    else:
        slabs = [Slab(n, precision=a.precision, rank=r, nranks=a.ranks) for r in range(a.ranks)]
        vs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in v] for r, s in enumerate(slabs)]
        fs = [[x[s.ista[r]:s.ista[r] + s.nxhl[r]].clone() for x in f] for r, s in enumerate(slabs)]
        del v, f, g
        step = lambda k: run_local(slabs, k, 4, dt, nu, vs, fs)
        ranks = a.ranks
    step(a.warmup)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    step(a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"workload": f"slab-decomposed forced HD {n}^3, RK4, {a.precision}, {ranks} ranks"
                                      + (" over NCCL" if world > 1 else " in one process on one GPU"),
                          "steps": a.steps, "ms_per_step": ms, "steps_per_s": 1000.0 / ms, "ranks": ranks,
                          "n_gpus": world}))


if __name__ == "__main__":
    main()
