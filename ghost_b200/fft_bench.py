"""Timing of the plain 3D transforms (fftp3d_real_to_complex and
fftp3d_complex_to_real) with the library's per-pass CUDA-event timers.

    python -m ghost_b200.fft_bench [--shape 512,512,512] [--reps 10] [--precision fp32]

One warm-up pair, then `reps` pairs of r2c + c2r on a seeded real field.
Prints one JSON line: per pass the mean time per launch and GB/s, counting
one read and one write of the whole field per pass (x: real + complex, y and
z: two complex fields).
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", default="512,512,512")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    a = ap.parse_args(argv)

    import torch

    from ghost_b200 import GHOST_COMPLEX_TO_REAL, GHOST_REAL_TO_COMPLEX, Ghost

    nx, ny, nz = (int(v) for v in a.shape.split(","))
    g = Ghost(nx, ny, nz, precision=a.precision)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    r = torch.randn(g.rshape, device="cuda", generator=gen, dtype=g.rtorch)
    c = g.czeros()
    fwd = g.fftp3d_create_plan((nx, ny, nz), GHOST_REAL_TO_COMPLEX)
    inv = g.fftp3d_create_plan((nx, ny, nz), GHOST_COMPLEX_TO_REAL)
    g.fftp3d_real_to_complex(fwd, r, c)
    g.fftp3d_complex_to_real(inv, c, r)
    torch.cuda.synchronize()
    g.enable_timers(True)
    g.read_timers()
    for _ in range(a.reps):
        g.fftp3d_real_to_complex(fwd, r, c)
        g.fftp3d_complex_to_real(inv, c, r)
    torch.cuda.synchronize()
    tm = g.read_timers()
    es = 4 if a.precision == "fp32" else 8
    R = nx * ny * nz * es
    C = (nx // 2 + 1) * ny * nz * 2 * es
    out = {}
    for k, (t, n) in tm.items():
        if not n:
            continue
        nbytes = R + C if k.startswith("x_") else 2 * C
        ms = t / n
        out[k] = {"ms_per_launch": ms, "launches": n, "gbs": nbytes / (ms * 1e-3) / 1e9}
    print(json.dumps({"shape": [nx, ny, nz], "precision": a.precision, "reps": a.reps, "passes": out}))
    g.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
