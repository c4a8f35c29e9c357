"""Timing of the subgrid-stress network's kernels on seeded inputs.

    python -m ghost_b200.mlp_bench [--rows 2097152] [--batch 65536] [--reps 20]

Forward over `rows` points (one LES evaluation at 128^3 is 2,097,152 rows)
and training steps (forward, backward, Adam) on batches of `batch`.  Prints
one JSON line with ms per call, rows/s and the tensor-core FLOP rate
(2 x (10x64 + 64x64 + 64x6) FLOPs per row forward; the backward adds the two
data products and the weight-gradient sums).
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=128 ** 3)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)

    import torch

    from ghost_b200.les import MLP

    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    x = torch.randn((a.rows, 10), generator=g, device="cuda")
    y = torch.empty((a.rows, 6), device="cuda")
    xb = x[: a.batch].contiguous()
    tb = torch.randn((a.batch, 6), generator=g, device="cuda")
    m = MLP(3)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0.record(s)
        for _ in range(a.reps):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / a.reps

    fwd = timed(lambda: m.forward(x, y))
    trn = timed(lambda: m.train_step(xb, tb, 1e-4, want_loss=False))
    flops_row = 2 * (10 * 64 + 64 * 64 + 64 * 6)
    print(json.dumps({
        "forward": {"rows": a.rows, "ms": fwd, "rows_per_s": a.rows / (fwd * 1e-3),
                    "tflops": flops_row * a.rows / (fwd * 1e-3) / 1e12},
        "train_step": {"batch": a.batch, "ms": trn, "rows_per_s": a.batch / (trn * 1e-3)},
    }))
    m.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
