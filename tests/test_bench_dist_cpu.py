"""The bench's multi-rank path on CPU with world_size 2 over gloo: ranks
advance different seeded batches, time is the max over ranks, the reported
value aggregates all ranks (weak scaling), and the reference arm runs and
prints on rank 0 only."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        el_ms = 10.0 + 5.0 * rank  # per-rank device time
        m = bench.max_over_ranks(dist, el_ms, device="cpu")
        X = np.linspace(-1, 1, 8)[None, :]
        P = np.linspace(-1, 1, 8)[:, None]
        W = bench.initial_states(np.random.default_rng(1000 + rank), 2, X, P)
        checksum = torch.tensor([float(W.sum())], dtype=torch.float64)
        gathered = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, checksum)
        out[rank] = (m, bench.job_value(100, 10, world, m), [float(g) for g in gathered])
    finally:
        dist.destroy_process_group()


def test_weak_scaling_aggregation_over_two_gloo_ranks():
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(2, free_port(), out), nprocs=2, join=True)
    for r in range(2):
        m, v, sums = out[r]
        assert m == 15.0  # max over ranks, on every rank
        assert abs(v - 100 * 10 * 2 / 15e-3) < 1e-6
        assert sums[0] != sums[1]  # each rank advances its own seeded batch


def test_reference_arm_prints_on_rank_zero_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"),
           "--gpus", "2", "--impl", "reference", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
