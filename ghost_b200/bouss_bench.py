"""Rotating stratified Boussinesq benchmark (the ROTBOUSS step on an
elongated box), GHOST's bench=1 style.

    python -m ghost_b200.bouss_bench [--shape 1024,1024,256] [--steps 10] [--precision fp32]

Workload: box 2pi x 2pi x pi/2 (ARBSIZE, Lx = Ly = 1, Lz = 1/4 in units of
2pi), seeded random solenoidal velocity on the shells 2 <= |k| <= 4 with
<|v|^2> = 1 (energy peaked near k = 3), zero temperature perturbation,
Brunt-Vaisala frequency N = 8 (xmom = xtemp = 8), rotation f = 1 about z
(omegaz = 0.5), nu = kappa = 5e-4, RK4, dt = 2.5e-4.  Prints one JSON line:
steps/s, ms per step, the per-pass split from the library's timers and the
energy before and after.
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", default="1024,1024,256")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    a = ap.parse_args(argv)

    import torch

    from ghost_b200 import Ghost

    nx, ny, nz = (int(x) for x in a.shape.split(","))
    g = Ghost(nx, ny, nz, 1.0, 1.0, 0.25, arbsize=True, precision=a.precision)
    v = [g.czeros() for _ in range(3)]
    th = g.czeros()
    g.init_random_solenoidal(1000, 2.0, 4.0, 0, 1.0, *v)
    args = (4, 2.5e-4, 5e-4, 5e-4, 0.5, 8.0, 8.0)
    e_start = g.energy(*v, 1)
    for _ in range(a.warmup):
        g.bouss_run(1, *args, *v, th)
    torch.cuda.synchronize()
    g.enable_timers(True)
    g.read_timers()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    g.bouss_run(a.steps, *args, *v, th)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    tm = g.read_timers()
    print(json.dumps({
        "workload": f"rotating stratified Boussinesq {nx}x{ny}x{nz}, box 2pi x 2pi x pi/2, RK4, dt=2.5e-4, "
                    f"N=8, f=1, nu=kappa=5e-4, {a.precision}",
        "steps": a.steps, "ms_per_step": ms / a.steps, "steps_per_s": a.steps / (ms * 1e-3),
        "passes_ms_per_step": {k: t / a.steps for k, (t, n) in tm.items() if n},
        "energy_start": e_start, "energy_end": g.energy(*v, 1), "tile_cfg": g.tile_cfg(),
    }))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
