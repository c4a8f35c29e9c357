"""GHOST's benchmark mode (bench=1, main3D.fpp:2521-2537, 3423-3483) for the
B200 library: advance the HD solver a number of RK steps from the seeded
initial condition and report per-step wall time and per-kernel device time.

    python -m ghost_b200.hd_bench --n 512 --steps 10 --precision fp32 [--out benchmark.txt]
    python -m ghost_b200.hd_bench --shape 512,512,64 ...    # a slab of the 512^3 passes

A non-cubic --shape keeps the x and y lines of the cubic run at a fraction of
its memory (the 2/3 truncation then follows GHOST's anisotropic kn2); it is
the size used for multi-pass profiler captures of the 512-point passes.

The output file follows benchmark.txt's spirit: grid, steps, then seconds
per step (device) and the per-pass split measured with the library's
kernel timers.
"""
from __future__ import annotations

import argparse
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--shape", default=None, help="nx,ny,nz (overrides --n)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--ord", type=int, default=4)
    ap.add_argument("--dt", type=float, default=5e-4)
    ap.add_argument("--nu", type=float, default=1e-3)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--tile-cfg", type=int, default=None, help="tile variant; default: autotune")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)

    import torch

    from ghost_b200 import Ghost

    nx, ny, nz = (int(x) for x in a.shape.split(",")) if a.shape else (a.n, a.n, a.n)
    g = Ghost(nx, ny, nz, precision=a.precision)
    v = [g.czeros() for _ in range(3)]
    f = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, min(nx, ny, nz) / 3.0, 1, 1.0, *v)
    g.init_random_solenoidal(2000, 2.0, 3.0, 0, 1.0, *f)
    if a.tile_cfg is None:
        cfg = g.hd_autotune(a.ord, a.dt, a.nu, *v, *f)
    else:
        g.set_tile_cfg(a.tile_cfg)
        cfg = a.tile_cfg
    for _ in range(a.warmup):
        g.hd_run(1, a.ord, a.dt, a.nu, *v, *f)
    torch.cuda.synchronize()
    g.enable_timers(True)
    g.read_timers()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(s)
    g.hd_run(a.steps, a.ord, a.dt, a.nu, *v, *f)
    e1.record(s)
    e1.synchronize()
    wall = time.perf_counter() - t0
    tm = g.read_timers()
    ms = e0.elapsed_time(e1)
    eng = g.energy(*v, 1)
    lines = [f"{nx} {ny} {nz} {a.steps} 1 {a.precision} {ms / 1e3 / a.steps:.6e} {wall / a.steps:.6e}"]
    for k, (t, n) in tm.items():
        lines.append(f"  {k:10s} {t / a.steps:9.3f} ms/step  {n // a.steps:3d} launches/step")
    lines.append(f"  <|v|^2> after run: {eng:.12e}")
    lines.append(f"  tile variant {cfg}")
    text = "\n".join(lines)
    print(text)
    if a.out:
        with open(a.out, "a") as fh:
            fh.write(text + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
