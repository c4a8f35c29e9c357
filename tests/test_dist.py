"""The N > 1 host path of bench.py on CPU: world_size-2 gloo process groups
(torchrun's environment, 127.0.0.1 rendezvous), the barrier, the max over
ranks used for timings, and the reference arm under torchrun (rank 0 alone
measures and prints one line; the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    import torch.distributed as dist
    ws_, rank_, _ = bench.dist_init(argparse.Namespace(impl="reference"))
    assert dist.get_backend() == "gloo"
    bench.barrier(ws_)
    m = bench.max_over_ranks(ws_, 1.5 + rank_)
    bench.barrier(ws_)
    with open(os.path.join(out, f"r{rank_}"), "w") as f:
        f.write(repr(m))
    dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert [float(open(tmp_path / f"r{r}").read()) for r in range(2)] == [2.5, 2.5]


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           "bench.py", "--impl", "reference", "--gpus", "2", "--grid", "32", "--steps", "2", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=500, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
    # --steps 2 substeps round up to one whole RK4 step, and the line's
    # steps, ms_per_step and value describe the same timed seconds
    assert d["steps"] == 1 and d["substeps_timed"] == 4 and d["steps_requested"] == 2
    assert abs(d["steps"] * d["ms_per_step"] * 1e-3 - d["steps"] / d["value"]) < 1e-9


def test_ensemble_shards_partition_the_runs():
    """The ensemble's shards (runs sharded by index, no communication): every
    run belongs to exactly one rank, class by class, with balanced counts."""
    from ghost_b200.ensemble_bench import shard_runs
    runs = [128, 96, 32]
    for world in (1, 2, 3, 4, 8):
        seen = []
        per = []
        for rank in range(world):
            counts, idx = shard_runs(runs, rank, world)
            assert sum(counts) == len(idx)
            per.append(counts)
            seen.extend(idx)
        assert sorted(seen) == list(range(sum(runs)))
        for c in range(len(runs)):
            col = [p[c] for p in per]
            assert max(col) - min(col) <= 1 and sum(col) == runs[c]


def _shard_worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from ghost_b200.ensemble_bench import shard_runs
    dist.init_process_group("gloo")
    _, idx = shard_runs([5, 4, 3], rank, ws)
    n = torch.tensor([len(idx)])
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(ws)]
    dist.all_gather(sizes, n)
    buf = torch.full((12,), -1, dtype=torch.int64)
    buf[:len(idx)] = torch.tensor(idx)
    gathered = [torch.zeros(12, dtype=torch.int64) for _ in range(ws)]
    dist.all_gather(gathered, buf)
    if rank == 0:
        allidx = sorted(int(v) for g in gathered for v in g.tolist() if v >= 0)
        with open(os.path.join(out, "idx"), "w") as f:
            f.write(repr(allidx))
    dist.destroy_process_group()


def test_ensemble_shards_under_gloo(tmp_path):
    """Two gloo ranks take their shards independently; together they hold
    every run once."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_shard_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert eval(open(tmp_path / "idx").read()) == list(range(12))
