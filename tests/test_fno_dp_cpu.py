"""Host side of data-parallel surrogate training on CPU with world_size 2 over
gloo: the flat-buffer gradient average, the common number of steps per epoch
when the ranks hold different numbers of samples, the split of the plain-Bloch
runs, and that averaged per-rank gradients of a mean loss equal the gradient
over the union of the ranks' batches (what keeps the replicas identical)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fastwigner_b200.fno import allreduce_mean_, dp_steps_per_epoch
from fastwigner_b200.surrogate import local_runs


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = dist.group.WORLD
        a = torch.full((3, 2), float(rank + 1))
        b = torch.arange(5, dtype=torch.float32) * (rank + 1)
        allreduce_mean_([a, b], g)
        steps = dp_steps_per_epoch([35, 50][rank], 8, g)
        # linear model y = x . w with mean squared loss: each rank's gradient
        # on its own batch, averaged, against the gradient on both batches
        rng = np.random.default_rng(0)
        X = torch.tensor(rng.normal(size=(16, 4)), dtype=torch.float64)
        Y = torch.tensor(rng.normal(size=16), dtype=torch.float64)
        w = torch.tensor(rng.normal(size=4), dtype=torch.float64)
        Xi, Yi = X[8 * rank:8 * rank + 8], Y[8 * rank:8 * rank + 8]
        grad = 2.0 * Xi.T @ (Xi @ w - Yi) / len(Yi)
        allreduce_mean_([grad], g)
        full = 2.0 * X.T @ (X @ w - Y) / len(Y)
        out[rank] = (a.numpy().copy(), b.numpy().copy(), steps, float((grad - full).abs().max()))
    finally:
        dist.destroy_process_group()


def test_gradient_average_and_common_steps_over_two_gloo_ranks():
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(2, free_port(), out), nprocs=2, join=True)
    for r in range(2):
        a, b, steps, gerr = out[r]
        np.testing.assert_array_equal(a, np.full((3, 2), 1.5, dtype=np.float32))
        np.testing.assert_array_equal(b, np.arange(5, dtype=np.float32) * 1.5)
        assert steps == 4  # min(35 // 8, 50 // 8) on both ranks
        assert gerr < 1e-12


def test_runs_split_over_ranks():
    for runs in (1, 7, 200):
        for world in (1, 2, 3, 8):
            parts = [local_runs(runs, world, r) for r in range(world)]
            assert sum(parts) == runs and max(parts) - min(parts) <= 1


def test_single_process_needs_no_group():
    assert dp_steps_per_epoch(35, 8, None) == 4
