#!/usr/bin/env python
"""Benchmark: HD 512^3 RK steps/s on B200, FP32 fast path vs FP64 plain path.

Workload (forced HD turbulence at 512^3): seeded random solenoidal velocity
with E(k) ~ k^4 exp(-2(k/2)^2) on 1 <= |k| <= N/3 normalised to <|v|^2> = 1,
constant random solenoidal forcing on 2 <= |k| <= 3 with f0 = 1, nu = 1e-3,
dt = 5e-4, RK order 4, 2/3 dealiasing.  A step is one full RK4 step (four
fused substeps).  Inputs (0.54 GB per FP32 field) are far larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times GHOST's CPU path on the host cores: the same steps
(fftp-3 transforms, prodre3, nonlhd3, the truncated update) with a threaded
library FFT, as GHOST's FFTW/OpenMP build runs them (GHOST itself needs
Fortran, MPI and FFTW, none of which exist here).  It times K RK substeps
rounded up to whole RK4 steps (ceil(K/4) steps, each timed whole) and
reports those steps, so that the run ends within minutes.
With torchrun (N > 1) the ranks advance ONE 512^3 run split into GHOST's
kx-slabs / z-slabs, with NCCL all-to-alls in field groups overlapped with the
Y passes (strong scaling; the plain schedule of one all-to-all per transform
direction is timed beside it); N = 1 runs the undivided fused step.

The e2e figure calls ghost_hd_run with pinned host arrays every step: the
library moves each array's live box (the kx rows, y-lines and kz values that
can hold a kept mode) and checks, on the host for the input and on the
device for the result, that the rest holds only zero bits.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HD 512³ RK steps/s, FP32 vs FP64 on 1 B200 (rel err ≤1e-5); FFT HBM %peak"
N = 512
ORD, DT, NU = 4, 5e-4, 1e-3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=N, help="cubic grid size (default 512)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"ghost_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        if not rows:
            return None
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def dist_init(args):
    """One process per GPU from torchrun's environment.  The GPU arm talks
    over NCCL; the reference arm (host cores only) and GPU-less hosts over
    gloo."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" and torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- CPU arm
def cpu_fields(o):
    v, _ = o.random_solenoidal(1000, 1.0, o.nx / 3.0, 1, 1.0)
    f, _ = o.random_solenoidal(2000, 2.0, 3.0, 0, 1.0)
    return v, f


def cpu_substep_times(n, samples, warmup, kind="fftlib", threads=None):
    """Seconds of each timed RK substep at n^3 FP32 on the host cores.
    kind "fftlib": GHOST's steps with a threaded library FFT (scipy's
    pocketfft, all host threads), the stand-in for its FFTW/OpenMP build;
    kind "oracle": the C restatement (OpenMP, its own textbook FFT)."""
    from oracle.oracle import Oracle
    o = Oracle(n, precision="fp32")
    v, f = cpu_fields(o)
    C = [x.copy() for x in v]
    if kind == "fftlib":
        from oracle.fftlib import FFTLibHD
        lib = FFTLibHD(o, threads)
        step, cores = lib.hd_rkstep2, lib.threads
    else:
        step, cores = o.hd_rkstep2, o.nthreads()
    times = []
    for s in range(warmup + samples):
        # timed substeps start a fresh RK step, so that timing ORD x m of
        # them times m whole RK steps (C = v at each step's start)
        o = ORD - ((s - warmup) % ORD if s >= warmup else s % ORD)
        if o == ORD:
            C = [x.copy() for x in v]
        t0 = time.perf_counter()
        v = step(o, DT, NU, v, C, f)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    if kind == "fftlib":
        lib.close()
    return times, cores


def run_reference(args, ws, rank):
    """GHOST's CPU path on the host cores.  A whole RK4 step of the CPU path
    takes ~10 s, so K of them would not fit the run: the arm times K RK
    substeps rounded up to whole RK4 steps (ceil(K/4) steps, each its four
    substeps in GHOST's order) after W untimed substeps, and reports those
    RK4 steps: "steps" = ceil(K/4), ms_per_step = mean RK4 step time,
    value = RK4 steps/s."""
    if rank != 0:
        return
    n_rk = max(1, -(-args.steps // ORD))
    times, cores = cpu_substep_times(args.grid, ORD * n_rk, max(0, args.warmup))
    t = sum(times) / n_rk
    val = 1.0 / t
    sample = (f"{n_rk} whole RK{ORD} steps ({ORD * n_rk} substeps; --steps {args.steps} asked for that many "
              f"substeps, rounded up to whole steps) at {args.grid}^3 FP32 of GHOST's CPU path with a threaded "
              f"library FFT (scipy pocketfft, {cores} threads), after {args.warmup} untimed substeps; "
              f"value = RK{ORD} steps / timed seconds")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": n_rk, "warmup": args.warmup, "ms_per_step": 1e3 * t, "substeps_timed": ORD * n_rk,
            "steps_requested": args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"HD forced turbulence {args.grid}^3, RK{ORD}, dt={DT}, nu={NU}, FP32",
                       "runs": "GHOST's fftp-3 + pseudospec3D_hd steps on the host cores, scipy.fft (pocketfft) "
                               "in place of FFTW, numpy elementwise work split over the same threads",
                       "step": f"one whole RK{ORD} step ({ORD} substeps); warmup counts substeps"},
            "cpu_baseline": {"value": val, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def setup_run(n, prec, rank):
    from ghost_b200 import Ghost
    g = Ghost(n, precision=prec)
    v = [g.czeros() for _ in range(3)]
    f = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000 + rank, 1.0, n / 3.0, 1, 1.0, *v)
    g.init_random_solenoidal(2000 + rank, 2.0, 3.0, 0, 1.0, *f)
    # the library's tile autotuner (FFTW's planner plays this role in GHOST),
    # on a copy of the state and outside the timed region
    g.tile = g.hd_autotune(ORD, DT, NU, *v, *f)
    return g, v, f


def timed_steps(g, v, f, steps, warmup, ws, timers=False):
    import torch
    for _ in range(warmup):
        g.hd_run(1, ORD, DT, NU, *v, *f)
    stream = torch.cuda.current_stream()
    barrier(ws)
    torch.cuda.synchronize()
    if timers:
        g.enable_timers(True)
        g.read_timers()
    n0 = g.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.hd_run(steps, ORD, DT, NU, *v, *f)
    e1.record(stream)
    e1.synchronize()
    launches = g.launch_count() - n0
    ms = e0.elapsed_time(e1)
    tm = g.read_timers() if timers else None
    if timers:
        g.enable_timers(False)
    torch.cuda.synchronize()
    barrier(ws)
    return max_over_ranks(ws, ms), launches, tm


def rel_err_fp32_step(n, rank):
    """FP32 step against the FP64 step from the same state (relative L2)."""
    import torch
    g64, v64, f64 = setup_run(n, "fp64", rank)
    g64.hd_run(2, ORD, DT, NU, *v64, *f64)  # develop the state
    g32, v32, f32 = setup_run(n, "fp32", rank)
    for a, b in zip(v32, v64):
        a.copy_(b.to(torch.complex64))
    for a, b in zip(f32, f64):
        a.copy_(b.to(torch.complex64))
    errs = []
    for _ in range(2):
        g64.hd_run(1, ORD, DT, NU, *v64, *f64)
        g32.hd_run(1, ORD, DT, NU, *v32, *f32)
        num = sum(float(torch.sum(torch.abs(a.to(torch.complex128) - b) ** 2)) for a, b in zip(v32, v64))
        den = sum(float(torch.sum(torch.abs(b) ** 2)) for b in v64)
        errs.append((num / den) ** 0.5)
        for a, b in zip(v32, v64):  # restart from the FP64 state: per-step error
            a.copy_(b.to(torch.complex64))
    g64.close()
    g32.close()
    del v64, f64, v32, f32
    torch.cuda.empty_cache()
    return max(errs)


def fft_roofline(n, peak, reps=10):
    """Standalone 3D r2c and c2r at n^3 FP32.  Whole transform: achieved
    (R + C) bytes / time.  Per pass (the kernels): every pass reads and
    writes the whole field once (x: R + C, y and z: 2C), against the
    library's own per-pass CUDA-event timers."""
    import torch
    from ghost_b200 import GHOST_COMPLEX_TO_REAL, GHOST_REAL_TO_COMPLEX, Ghost
    g = Ghost(n, precision="fp32")
    x = torch.randn((n, n, n), device="cuda", dtype=torch.float32)
    c = g.czeros()
    fwd = g.fftp3d_create_plan((n, n, n), GHOST_REAL_TO_COMPLEX)
    inv = g.fftp3d_create_plan((n, n, n), GHOST_COMPLEX_TO_REAL)
    R = n ** 3 * 4
    C = (n // 2 + 1) * n * n * 8
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        g.enable_timers(True)
        g.read_timers()
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        e1.synchronize()
        tm = g.read_timers()
        g.enable_timers(False)
        return e0.elapsed_time(e1) / reps, tm

    ms_f, tm_f = timed(lambda: g.fftp3d_real_to_complex(fwd, x, c))
    ms_i, tm_i = timed(lambda: g.fftp3d_complex_to_real(inv, c, x))
    g.close()
    del x, c
    torch.cuda.empty_cache()
    passes = {}
    for tm in (tm_f, tm_i):
        for k, (t, cnt) in tm.items():
            if not cnt:
                continue
            nbytes = R + C if k.startswith("x_") else 2 * C
            ms = t / cnt
            passes[k] = {"ms_per_launch": ms, "bytes": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9,
                         "frac": nbytes / (ms * 1e-3) / 1e9 / peak}
    return {"ms_per_fft": ms_f, "ms_per_ifft": ms_i, "algorithmic_bytes": R + C,
            "gbs": (R + C) / (ms_f * 1e-3) / 1e9, "frac": (R + C) / (ms_f * 1e-3) / 1e9 / peak,
            "passes": passes, "min_pass_frac": min(p["frac"] for p in passes.values())}


def e2e_host(n, steps, rank):
    """Through the public C ABI with pinned host arrays: every step copies
    the velocity and forcing in and the velocity out (GHOST's host-array
    calling convention).  The library moves the live box of each array (the
    kx rows and y-lines that hold kept modes): the forcing's in (it is never
    read elsewhere), the velocity's in (host threads find only zero bits
    outside the box, so the device copy is zeroed there instead) and the
    velocity's out (the result holds only zero bits outside the box, checked
    on the device).  Any nonzero bit outside the box moves the whole array.
    The byte counts are the moves of this run, checked below."""
    import torch
    from ghost_b200 import Ghost
    g, v, f = setup_run(n, "fp32", rank)
    hv = [torch.empty(g.sshape, dtype=torch.complex64, pin_memory=True) for _ in range(3)]
    hf = [torch.empty(g.sshape, dtype=torch.complex64, pin_memory=True) for _ in range(3)]
    for a, b in zip(hv, v):
        a.copy_(b)
    for a, b in zip(hf, f):
        a.copy_(b)
    del v, f
    torch.cuda.empty_cache()
    nv = [x.numpy() for x in hv]
    nf = [x.numpy() for x in hf]
    g.hd_run(1, ORD, DT, NU, *nv, *nf)  # warm-up: staging buffers
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        g.hd_run(1, ORD, DT, NU, *nv, *nf)
    dt = time.perf_counter() - t0
    from ghost_b200.roofline import live_box
    live, jt, jb, kt, kb = live_box(n)
    zt, zb = (kt * 8 + 15) // 16 * 2, (kb * 8 + 15) // 16 * 2  # z blocks rounded out to 16-byte words
    dead = [int((x[live:] != 0).any() or (x[:live, jt:g.ny - jb] != 0).any()
                or (x[:live, :jt, zt:g.nz - zb] != 0).any() or (x[:live, g.ny - jb:, zt:g.nz - zb] != 0).any())
            for x in nv]
    g.close()
    if any(dead):
        raise RuntimeError("the velocity holds values outside the live box")
    box = live * (jt + jb) * (zt + zb) * 8
    return steps / dt, 6 * box, 3 * box


def traffic_from_profiles(kernel):
    """dram bytes per launch recorded from an ncu capture, if committed."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        p = line.split()
        if len(p) >= 2 and p[0] == kernel:
            try:
                return float(p[1])
            except ValueError:
                return None
    return None


def prune_fractions(n):
    """(f_line, f_row, f_keep) of the pruned passes (ghost_b200.roofline)."""
    from ghost_b200.roofline import prune_fractions as pf
    return pf(n)


def fp64_vs_cpu_oracle(g64, v64, f64):
    """One RK4 step of the FP64 plain path at full size (the first substep
    full, the other three zero-pruned, as timed) against the same step of the
    CPU FP64 oracle from the same state: relative L2 of v."""
    import numpy as np
    import torch

    from oracle.oracle import Oracle
    o = Oracle(g64.nx, g64.ny, g64.nz, precision="fp64")
    hv = [x.cpu().numpy() for x in v64]
    hf = [x.cpu().numpy() for x in f64]
    g64.hd_run(1, ORD, DT, NU, *v64, *f64)
    torch.cuda.synchronize()
    ref = o.hd_run(1, ORD, DT, NU, hv, hf)
    del hv, hf
    num = den = 0.0
    for a, b in zip(v64, ref):
        d = a.cpu().numpy()
        num += float(np.sum(np.abs(d - b) ** 2))
        den += float(np.sum(np.abs(b) ** 2))
    return (num / den) ** 0.5


def cpu_baselines(n):
    """The host-core rates beside the GPU line: GHOST's CPU path with the
    threaded library FFT (1 warm-up and 3 timed substeps) and the C oracle
    restatement (2 timed substeps), both FP32 on all host threads."""
    t_lib, cores = cpu_substep_times(n, 3, 1, "fftlib")
    t_or, cores_or = cpu_substep_times(n, 2, 0, "oracle")
    m_lib, m_or = sum(t_lib) / len(t_lib), sum(t_or) / len(t_or)
    cpu = {"value": 1.0 / (ORD * m_lib), "unit": "steps/s", "cores": cores, "kind": "port",
           "sample": f"{len(t_lib)} RK substeps at {n}^3 FP32 (1/{ORD} of an RK{ORD} step each) after 1 untimed, "
                     f"GHOST's CPU path with scipy pocketfft in place of FFTW on {cores} threads; "
                     f"steps/s = 1/({ORD} x mean substep time)",
           "oracle_c": {"value": 1.0 / (ORD * m_or), "unit": "steps/s", "cores": cores_or,
                        "sample": f"{len(t_or)} RK substeps of the C restatement (textbook FFT, OpenMP)"}}
    return cpu


def run_ours(args, ws, rank, local):
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        return run_slab(args, ws, rank, local)
    n = args.grid
    peak, peak_kind = peaks()
    clocks = Clocks(local)

    # FP32 fast path (headline)
    g32, v32, f32 = setup_run(n, "fp32", rank)
    clocks.start()
    ms32, launches, tm = timed_steps(g32, v32, f32, args.steps, args.warmup, ws, timers=True)
    tile32 = g32.tile
    # FP64 plain path, same workload
    g32.close()
    del v32, f32
    torch.cuda.empty_cache()
    g64, v64, f64 = setup_run(n, "fp64", rank)
    steps64_n = max(2, args.steps // 2)
    ms64, _, tm64 = timed_steps(g64, v64, f64, steps64_n, args.warmup, ws, timers=True)
    tile64 = g64.tile
    clk = clocks.stop()
    err64 = fp64_vs_cpu_oracle(g64, v64, f64) if not args.no_cpu_baseline else None
    g64.close()
    del v64, f64
    torch.cuda.empty_cache()

    steps32 = args.steps / (ms32 * 1e-3)
    steps64 = steps64_n / (ms64 * 1e-3)

    # dominant kernel and its roofline: algorithmic bytes per launch, the
    # bytes each pass must move once the known zeros of the 2/3 truncation
    # are skipped (f_line: live z-lines, f_row: live kx rows, f_keep: kept modes)
    cb = (n // 2 + 1) * n * n * 8
    f_line, f_row, f_keep = prune_fractions(n)
    per_launch_bytes = {"z_inv": (9 + 3 / ORD) * f_line * cb,
                        "y_inv": 6 * (f_line + f_row) * cb,
                        "x_nl": 9 * f_row * cb,
                        "y_fwd": 3 * (f_row + f_line) * cb,
                        "z_fwd": (6 * f_line + 9 * f_keep) * cb}
    dom = max(tm, key=lambda k: tm[k][0])
    dom_ms = tm[dom][0] / tm[dom][1]
    ach = per_launch_bytes[dom] / (dom_ms * 1e-3) / 1e9

    def kern_table(t, scale):
        return {k: {"ms_per_launch": t[k][0] / t[k][1], "launches": t[k][1],
                    "share": t[k][0] / sum(x[0] for x in t.values()),
                    "gbs": scale * per_launch_bytes[k] / (t[k][0] / t[k][1] * 1e-3) / 1e9
                    if k in per_launch_bytes else None}
                for k in t}

    err = rel_err_fp32_step(n, rank)
    fft = fft_roofline(n, peak)
    e2e_val, h2d, d2h = e2e_host(n, args.e2e_steps, rank)
    cpu = cpu_baselines(n) if not args.no_cpu_baseline else None

    # algorithmic bytes per substep on the unpruned count 9 FFTs x (R + C) + 15 C
    R = n ** 3 * 4
    unpruned_bytes = 9 * (R + cb) + 15 * cb
    line = {
        "metric": METRIC, "value": steps32, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"HD forced turbulence {n}^3, RK{ORD}, dt={DT}, nu={NU}, FP32 fast path",
                   "parallelism": "single GPU",
                   "l2": "inputs larger than L2 (0.54 GB per FP32 field)"},
        "fp64": {"value": steps64, "unit": "steps/s", "ms_per_step": ms64 / steps64_n,
                 "tile_cfg": tile64, "kernels": kern_table(tm64, 2.0)},
        "tile_cfg": tile32,
        "fp32_over_fp64": steps32 / steps64,
        "fp32_rel_err_per_step": err,
        "fp64_rel_err_vs_cpu_oracle": err64,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "peak_kind": peak_kind,
                     "traffic": traffic_from_profiles(dom)},
        "kernels": kern_table(tm, 1.0),
        "fft": fft,
        "substep_effective_gbs": unpruned_bytes / (ms32 / args.steps / ORD * 1e-3) / 1e9,
        "prune": {"f_line": f_line, "f_row": f_row, "f_keep": f_keep},
        "substep_bytes": sum(per_launch_bytes.values()),
        "e2e": {"value": e2e_val, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_slab(args, ws, rank, local):
    """N > 1: one n^3 run split over the ranks in GHOST's slab layout
    (kx-slabs of the spectral fields, z-slabs for the x pass), NCCL
    all-to-alls per substep in field groups overlapped with the Y passes
    (ghost_b200.slab; the plain schedule of two all-to-alls per substep is
    timed beside it).  Every rank generates the
    same seeded fields as the one-GPU run and keeps its kx-slab."""
    import torch

    from ghost_b200 import Ghost
    from ghost_b200.roofline import slab_roofline
    from ghost_b200.slab import Slab
    n = args.grid
    clocks = Clocks(local)

    def setup(prec):
        g = Ghost(n, precision=prec)
        v = [g.czeros() for _ in range(3)]
        f = [g.czeros() for _ in range(3)]
        g.init_random_solenoidal(1000, 1.0, n / 3.0, 1, 1.0, *v)
        g.init_random_solenoidal(2000, 2.0, 3.0, 0, 1.0, *f)
        s = Slab(n, precision=prec, rank=rank, nranks=ws)
        lo, cnt = s.ista[rank], s.nxhl[rank]
        vs = [x[lo:lo + cnt].clone() for x in v]
        fs = [x[lo:lo + cnt].clone() for x in f]
        g.close()
        del v, f
        torch.cuda.empty_cache()
        return s, vs, fs

    def timed(s, vs, fs, steps, warmup):
        s.run(warmup, ORD, DT, NU, *vs, *fs)
        barrier(ws)
        torch.cuda.synchronize()
        n0 = s.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.run(steps, ORD, DT, NU, *vs, *fs)
        e1.record()
        e1.synchronize()
        launches = s.launch_count() - n0
        ms = max_over_ranks(ws, e0.elapsed_time(e1))
        barrier(ws)
        return ms, launches

    s32, v32, f32 = setup("fp32")
    clocks.start()
    ms32, launches = timed(s32, v32, f32, args.steps, args.warmup)
    # the plain schedule (one synchronous all-to-all per direction, own block
    # through the buffers) for comparison, and its exchange time per substep
    # (an extra step with events around the all-to-alls)
    s32.set_overlap(False)
    ms32_plain, _ = timed(s32, v32, f32, args.steps, 1)
    ev = []
    s32.run(1, ORD, DT, NU, *v32, *f32, exchange_events=ev)
    torch.cuda.synchronize()
    xch = max_over_ranks(ws, sum(a.elapsed_time(b) for a, b in ev) / ORD)
    barrier(ws)
    s32.set_overlap(True)
    # e2e: every step copies this rank's slabs of v and f in from pinned host
    # memory and v out, around the same library calls
    hv = [torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for x in v32]
    hf = [torch.empty(x.shape, dtype=x.dtype, pin_memory=True) for x in f32]
    for a, b in zip(hv + hf, v32 + f32):
        a.copy_(b)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.e2e_steps):
        for a, b in zip(v32 + f32, hv + hf):
            a.copy_(b, non_blocking=True)
        s32.run(1, ORD, DT, NU, *v32, *f32)
        for a, b in zip(hv, v32):
            a.copy_(b, non_blocking=True)
    e1.record()
    e1.synchronize()
    ms_e2e = max_over_ranks(ws, e0.elapsed_time(e1))
    cb_loc = v32[0].numel() * v32[0].element_size()
    tot = torch.tensor([6.0 * cb_loc, 3.0 * cb_loc], dtype=torch.float64, device="cuda")
    import torch.distributed as dist
    dist.all_reduce(tot)
    h2d, d2h = int(tot[0].item()), int(tot[1].item())
    s32.close()
    del v32, f32, hv, hf
    torch.cuda.empty_cache()
    s64, v64, f64 = setup("fp64")
    steps64_n = max(2, args.steps // 2)
    ms64, _ = timed(s64, v64, f64, steps64_n, args.warmup)
    clk = clocks.stop()
    s64.close()
    steps32 = args.steps / (ms32 * 1e-3)
    steps64 = steps64_n / (ms64 * 1e-3)
    if rank == 0:
        line = {
            "metric": METRIC, "value": steps32, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": f"HD forced turbulence {n}^3, RK{ORD}, dt={DT}, nu={NU}, FP32 fast path, one run "
                                   f"split over {ws} GPUs",
                       "parallelism": f"slab x{ws} (kx-slabs / z-slabs, NCCL all-to-all per transform direction)",
                       "l2": "inputs larger than L2"},
            "fp64": {"value": steps64, "unit": "steps/s", "ms_per_step": ms64 / steps64_n},
            "fp32_over_fp64": steps32 / steps64,
            "exchange_ms_per_substep": xch,
            "schedule": "overlapped: v and curl v exchanged as two asynchronous all-to-alls, the products one field "
                        "at a time, each behind the Y passes of the others; own block copied field to field",
            "plain_schedule_ms_per_step": ms32_plain / args.steps,
            "roofline": slab_roofline(n, ws, ms32 / args.steps, xch, ORD),
            "e2e": {"value": args.e2e_steps / (ms_e2e * 1e-3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches * ws,
            "gpu_launches_per_rank": launches,
            "clocks": clk,
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
