"""Ensemble throughput: 256 independent HD runs of uneven sizes advanced
together (one batched context per size, one RK step of all of them replayed
as a CUDA graph, tile shapes from the autotuner).

    python -m ghost_b200.ensemble_bench [--steps 500] [--precision fp32]

Default workload: 128 runs at 32^3, 96 at 64^3, 32 at 128^3 (96.5M grid
points), seeds 1000+r, nu log-uniform in [5e-4, 5e-3] from a seeded host
RNG, the config-0 initial spectrum, RK2, dt = 1e-3.  Prints one JSON line
with run-steps/s and grid-point-steps/s.
"""
from __future__ import annotations

import argparse
import json
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="32,64,128")
    ap.add_argument("--runs", default="128,96,32")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--ord", type=int, default=2)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    a = ap.parse_args(argv)

    import numpy as np
    import torch

    from ghost_b200 import Ensemble

    sizes = [int(x) for x in a.sizes.split(",")]
    runs = [int(x) for x in a.runs.split(",")]
    total = sum(runs)
    rng = np.random.default_rng(20261203)
    nu = np.exp(rng.uniform(np.log(5e-4), np.log(5e-3), total))
    seeds = [1000 + r for r in range(total)]
    t0 = time.perf_counter()
    ens = Ensemble(sizes, runs, precision=a.precision)
    ens.init(seeds, nu)
    cfg = ens.autotune(a.ord, a.dt)
    setup = time.perf_counter() - t0
    ens.run(1, a.ord, a.dt)  # uncaptured first step, graph capture
    ens.run(1, a.ord, a.dt)
    torch.cuda.synchronize()
    e0 = ens.energy(1)
    t1 = time.perf_counter()
    ens.run(a.steps, a.ord, a.dt)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t1
    e1 = ens.energy(1)
    points = sum(r * n ** 3 for n, r in zip(sizes, runs))
    print(json.dumps({
        "workload": f"ensemble {'+'.join(f'{r}x{n}^3' for n, r in zip(sizes, runs))}, RK{a.ord}, dt={a.dt}, "
                    f"{a.precision}",
        "steps": a.steps, "seconds": wall, "run_steps_per_s": total * a.steps / wall,
        "ensemble_steps_per_s": a.steps / wall, "gridpoint_steps_per_s": points * a.steps / wall,
        "tile_cfg": cfg, "setup_s": setup,
        "energy_decay_min_max": [float((e1 / e0).min()), float((e1 / e0).max())],
    }))
    ens.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
