"""Ensemble throughput: 256 independent HD runs of uneven sizes advanced
together (one batched context per size, one RK step of all of them replayed
as a CUDA graph, tile shapes from the autotuner).

    python -m ghost_b200.ensemble_bench [--steps 500] [--precision fp32]
    torchrun --nproc-per-node N -m ghost_b200.ensemble_bench ...   # runs sharded over N GPUs

Under torchrun every rank advances its own share of the runs (round-robin
within each size class, with the seeds and viscosities of the whole
ensemble), with no communication; the time is the maximum over ranks and
the rates are those of the whole ensemble.

Two ways to run one substep of the ensemble are timed back to back (--mode
both, the default): "multi", each of the five passes one launch over all
size classes (a CTA picks its class from a per-class tile table), and
"per-class", each class's own launches on its own stream, with the tile
shapes the autotuner picked for that class.  The top-level rates are those
of the faster mode.

Default workload: 128 runs at 32^3, 96 at 64^3, 32 at 128^3 (96.5M grid
points), seeds 1000+r, nu log-uniform in [5e-4, 5e-3] from a seeded host
RNG, the config-0 initial spectrum, RK2, dt = 1e-3.  Prints one JSON line
with run-steps/s, grid-point-steps/s and the HBM roofline of the faster mode
(the pruned substeps' algorithmic bytes of every class, ghost_b200.roofline,
over the measured copy bandwidth).
"""
from __future__ import annotations

import argparse
import json
import time


def shard_runs(runs, rank, world):
    """Global run indices of this rank: run r of class c (runs numbered class
    by class) belongs to rank (r - first run of c) mod world.  Returns the
    per-class run counts of the shard and the global indices, class by class."""
    counts, idx, base = [], [], 0
    for r in runs:
        mine = [base + q for q in range(r) if q % world == rank]
        counts.append(len(mine))
        idx.extend(mine)
        base += r
    return counts, idx


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="32,64,128")
    ap.add_argument("--runs", default="128,96,32")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--ord", type=int, default=2)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--mode", default="both", choices=["both", "multi", "per-class"])
    a = ap.parse_args(argv)

    import numpy as np
    import torch

    from ghost_b200 import Ensemble

    import os
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    sizes = [int(x) for x in a.sizes.split(",")]
    runs = [int(x) for x in a.runs.split(",")]
    total = sum(runs)
    rng = np.random.default_rng(20261203)
    nu = np.exp(rng.uniform(np.log(5e-4), np.log(5e-3), total))
    seeds = [1000 + r for r in range(total)]
    counts, mine = shard_runs(runs, rank, world)
    keep = [q for q, c in enumerate(counts) if c > 0]
    t0 = time.perf_counter()
    ens = Ensemble([sizes[q] for q in keep], [counts[q] for q in keep], precision=a.precision)
    ens.init([seeds[r] for r in mine], nu[mine])
    cfg = ens.autotune(a.ord, a.dt)
    tuned_mode = "multi" if ens.mode() else "per-class"
    setup = time.perf_counter() - t0
    e0 = None
    modes = {"both": ["multi", "per-class"], "multi": ["multi"], "per-class": ["per-class"]}[a.mode]
    timing = {}
    for m in modes:
        try:
            ens.set_mode(m == "multi")
        except RuntimeError:
            if a.mode == "multi":
                raise
            continue  # classes outside the multi-class launches: per-class only
        ens.run(1, a.ord, a.dt)  # uncaptured first step, graph capture
        ens.run(1, a.ord, a.dt)
        torch.cuda.synchronize()
        if e0 is None:
            e0 = ens.energy(1)
        s = torch.cuda.current_stream()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(s)
        ens.run(a.steps, a.ord, a.dt)
        ev1.record(s)
        ev1.synchronize()
        wall = ev0.elapsed_time(ev1) * 1e-3
        if world > 1:
            t = torch.tensor([wall], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        timing[m] = wall
    e1 = ens.energy(1)
    points = sum(r * n ** 3 for n, r in zip(sizes, runs))
    best = min(timing, key=timing.get)
    wall = timing[best]
    # HBM roofline: the pruned substep's algorithmic bytes of every class (no forcing)
    from ghost_b200.roofline import measured_hbm_peak, pass_bytes
    eb = 8 if a.precision == "fp32" else 16
    step_bytes = a.ord * sum(sum(pass_bytes(n, a.ord, False, eb, r).values()) for n, r in zip(sizes, runs))
    peak, peak_kind = measured_hbm_peak()
    achieved = step_bytes * a.steps / wall / 1e9
    if rank == 0:
        print(json.dumps({
            "workload": f"ensemble {'+'.join(f'{r}x{n}^3' for n, r in zip(sizes, runs))}, RK{a.ord}, dt={a.dt}, "
                        f"{a.precision}",
            "gpus": world, "steps": a.steps, "seconds": wall, "run_steps_per_s": total * a.steps / wall,
            "ensemble_steps_per_s": a.steps / wall, "gridpoint_steps_per_s": points * a.steps / wall,
            "mode": best, "autotuned_mode": tuned_mode,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "bytes_per_ensemble_step": step_bytes},
            "modes": {m: {"seconds": w, "run_steps_per_s": total * a.steps / w,
                          "gridpoint_steps_per_s": points * a.steps / w} for m, w in timing.items()},
            "tile_cfg": cfg, "setup_s": setup,
            "energy_decay_min_max": [float((e1 / e0).min()), float((e1 / e0).max())],
        }))
    ens.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
