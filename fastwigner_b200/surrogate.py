"""Train the FNO surrogate on plain-Bloch thermal states and measure what it
gains: wall time to a thermal state with and without the surrogate seed.

    python -m fastwigner_b200.surrogate [--runs 1000] [--nbeta 20] [--epochs 10] [--out results.json]
    torchrun --nproc-per-node N -m fastwigner_b200.surrogate --dp ...   # data-parallel training
    python -m fastwigner_b200.surrogate --time-network [--reps 5]          # network timings only

The workload is the Morse-oscillator thermal-state problem
(V = D (1 - exp(-a (x - x_e)))^2, D ~ U(2, 10), a ~ U(0.5, 1.5),
training states at beta log-spaced in [2, 20], dbeta = 1e-3, 512^2 FP32).  Error is measured with the
reference's own metric for thermal states, max |W - W_plain| dX dP
(wigner_bloch_fftw_1d.py:165-167), against the plain Bloch run from W = const
on the same GPU; both runs are timed with CUDA events.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .benchmarks import ClockSampler
from .fno import BlochBatch, BlochSurrogate, FNO2d, MorseBlochSetup, generate_dataset


def timed(fn):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def local_runs(runs, world, rank):
    """Plain-Bloch runs generated by `rank` when `runs` are shared by `world`
    data-parallel ranks (the first runs % world ranks take one more)."""
    return runs // world + (1 if rank < runs % world else 0)


def run_study(runs=1000, nbeta=20, epochs=10, batch=16, grid=512, train_grid=512, eval_betas=(5.0, 10.0, 20.0),
              n_eval=16, refine_fraction=0.05, seed=0, width=32, modes=(16, 16), layers=4, lr=2e-3,
              residual=True, log=print, group=None, beta_range=(2.0, 20.0), min_refine=0.25, save=None, load=None):
    """group: a process group for data-parallel training -- each rank
    generates its share of the runs (its own seed), the network starts from
    the same seed everywhere and the gradients are averaged before every step;
    rank 0 alone evaluates and returns the results (the others return None).
    save / load: an .npz of the trained network's parameters; with `load` the
    data generation and training are skipped."""
    world, rank = 1, 0
    if group is not None:
        import torch.distributed as dist

        world, rank = dist.get_world_size(group), dist.get_rank(group)
    rng = np.random.default_rng(seed + 7919 * rank)
    setup = MorseBlochSetup(grid=grid)
    betas = np.exp(np.linspace(np.log(beta_range[0]), np.log(beta_range[1]), nbeta))
    net = FNO2d(n_params=3, width=width, modes=modes, layers=layers, proj=128, seed=seed)
    sur = BlochSurrogate(setup, net, train_grid=train_grid, residual=residual)
    t_data = t_train = 0.0
    losses, n_samples = [float("nan")], 0
    if load:
        net.load_state_dict(dict(np.load(load)))
    else:
        t0 = time.time()
        P, S = generate_dataset(setup, local_runs(runs, world, rank), betas, rng, train_grid=train_grid)
        t_data = time.time() - t0
        n_samples = int(len(P))
        t0 = time.time()
        losses = sur.train(P, S, epochs=epochs, batch=batch, lr=lr, rng=rng, group=group,
                           log=(lambda ep, l: log(f"epoch {ep}: loss {l:.3e}")) if (log and rank == 0) else None)
        torch.cuda.synchronize()
        t_train = time.time() - t0
        del P, S
        if save and rank == 0:
            np.savez(save, **net.state_dict())
    if rank != 0:
        return None
    dxdp = setup.dX * setup.dP
    results = []
    erng = np.random.default_rng(seed + 104729)  # held-out wells, the same whether trained here or loaded
    for beta in eval_betas:
        Ds = erng.uniform(2.0, 10.0, size=n_eval)
        As = erng.uniform(0.5, 1.5, size=n_eval)
        bb = BlochBatch(setup, Ds, As)  # exponent tables shared by both runs
        sur.predict(Ds[:1], As[:1], beta)  # warm-up (DFT matrices for the full grid)
        bb.set_uniform().run(2)
        with ClockSampler() as clk:
            (Wp, n_plain), ms_plain = timed(lambda: sur.plain_gibbs(bb, beta))
            Wp = Wp.clone()
            (Ws, n_seed), ms_seed = timed(lambda: sur.seeded_gibbs(bb, Ds, As, beta, refine_fraction=refine_fraction,
                                                                   min_refine=min_refine))
        err = ((Ws - Wp).abs().amax(dim=(1, 2)).double() * dxdp).cpu().numpy()
        seed_only = sur.predict(Ds, As, beta)  # the surrogate at beta itself, no refinement
        err_seed_only = ((seed_only - Wp).abs().amax(dim=(1, 2)).double() * dxdp).cpu().numpy()
        st = setup.G // train_grid  # the same error on the training points only
        err_seed_train = ((seed_only[:, ::st, ::st] - Wp[:, ::st, ::st]).abs().amax(dim=(1, 2)).double()
                          * dxdp).cpu().numpy()
        del bb
        results.append(dict(beta=beta, instances=n_eval, plain_steps=n_plain, seeded_steps=n_seed,
                            plain_ms=ms_plain, seeded_ms=ms_seed, speedup=ms_plain / ms_seed,
                            max_err=float(err.max()), median_err=float(np.median(err)),
                            surrogate_only_max_err=float(err_seed_only.max()),
                            surrogate_only_max_err_training_points=float(err_seed_train.max()),
                            clocks=clk.summary()))
        if log:
            log(json.dumps(results[-1]))
    return dict(data_seconds=t_data, train_seconds=t_train, final_loss=float(np.mean(losses[-50:])),
                samples=n_samples * world, loaded=load, ranks=world, epochs=epochs, residual=residual,
                train_grid=train_grid, width=width, modes=list(modes), refine_fraction=refine_fraction,
                min_refine=min_refine,
                beta_range=list(beta_range), results=results)


def time_network(grid=512, train_grid=256, n=16, reps=5, width=32, seed=0):
    """CUDA-event times (ms, mean of `reps` after one warm-up) of the
    surrogate's inference for `n` instances on the full grid and of one
    training step (forward, backward, Adam) on a batch of `n` at the training
    grid, with random weights and inputs."""
    setup = MorseBlochSetup(grid=grid)
    net = FNO2d(n_params=3, width=width, modes=(16, 16), layers=4, proj=128, seed=seed)
    sur = BlochSurrogate(setup, net, train_grid=train_grid)
    rng = np.random.default_rng(seed)
    Ds, As = rng.uniform(2.0, 10.0, n), rng.uniform(0.5, 1.5, n)
    X = rng.uniform(-1.0, 1.0, size=(n, 3))
    T = torch.zeros((n, train_grid, train_grid), dtype=torch.float32, device=net.device)

    def train_step():
        _, dY = net.loss_and_grad(X, sur.xs_t, sur.ps_t, T)
        net.backward(dY)
        net.adam_step(1e-4)

    out = {}
    for name, fn in ((f"predict_{n}x{grid}_ms", lambda: sur.predict(Ds, As, 4.0)),
                     (f"train_step_{n}x{train_grid}_ms", train_step)):
        fn()
        _, ms = timed(lambda: [fn() for _ in range(reps)])
        out[name] = ms / reps
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=1000)
    ap.add_argument("--nbeta", type=int, default=20)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--refine", type=float, default=0.05)
    ap.add_argument("--train-grid", type=int, default=512,
                    help="training grid (a subgrid of the 512^2 evaluation grid; the network is not resolution-invariant)")
    ap.add_argument("--width", type=int, default=32)
    ap.add_argument("--modes", type=int, default=16, help="retained Fourier modes along each axis")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--plain-target", action="store_true",
                    help="learn the thermal state itself instead of the correction to the harmonic baseline")
    ap.add_argument("--eval-betas", default="5,10,20")
    ap.add_argument("--beta-min", type=float, default=2.0, help="smallest recorded beta of the training data")
    ap.add_argument("--min-refine", type=float, default=0.25,
                    help="smallest beta interval refined by plain Bloch steps after the surrogate seed")
    ap.add_argument("--out", default=None)
    ap.add_argument("--dp", action="store_true",
                    help="data-parallel training, one process per GPU under torchrun (NCCL gradient all-reduce)")
    ap.add_argument("--save", default=None, help="write the trained network's parameters (.npz)")
    ap.add_argument("--load", default=None, help="evaluate a saved network (no data generation or training)")
    ap.add_argument("--time-network", action="store_true",
                    help="only time the network's inference and one training step (random weights), then exit")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    if a.time_network:
        print(json.dumps(time_network(train_grid=a.train_grid, reps=a.reps, width=a.width)))
        return
    group = None
    if a.dp:
        import datetime
        import os

        import torch.distributed as dist

        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        group = dist.group.WORLD
    try:
        r = run_study(runs=a.runs, nbeta=a.nbeta, epochs=a.epochs, refine_fraction=a.refine,
                      train_grid=a.train_grid, width=a.width, modes=(a.modes, a.modes), lr=a.lr,
                      residual=not a.plain_target,
                      eval_betas=tuple(float(b) for b in a.eval_betas.split(",")), group=group,
                      beta_range=(a.beta_min, 20.0), min_refine=a.min_refine, save=a.save, load=a.load)
    finally:
        if group is not None:
            import torch.distributed as dist

            dist.destroy_process_group()
    if r is not None:
        print(json.dumps(r))
        if a.out:
            with open(a.out, "w") as f:
                json.dump(r, f, indent=1)


if __name__ == "__main__":
    main()
