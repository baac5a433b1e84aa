#!/usr/bin/env python
"""Benchmark of the fused split-operator Moyal step (FP32 state, complex64
spectra, FP64-built phases) on the 1024 x 1024 anharmonic double-well
workload: V = 0.05 x^4 - x^2, K = p^2/2, X_amplitude = P_amplitude = 10,
dt = 0.005; every instance starts from a Gaussian wave packet with
x0 ~ U(-2, 2), p0 ~ U(-1, 1), width 0.5 (seeded).  A batch of instances is
advanced together so the states (B x 4 MiB) exceed the 126 MB L2: every pass
streams its tile from HBM.

One bench step = one time step of every instance of the batch (two fused
passes per instance).  value = grid-point steps per second over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload {moyal_fp64_256,vn_1024,bloch_512,batch_uneven,strong_field,
                                strong_field_frames,rho_to_wigner_1024,moyal_absorbing_1024}

Under torchrun (N > 1) every rank advances its own batch (different seeds,
no data-path collective): weak scaling, time = max over ranks.
``--impl reference`` times the reference algorithm's CPU path (the FP64
numpy restatement in oracle/, multi-threaded FFTs) on this host instead.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID = 1024
AMP = 10.0
DT = 0.005
WIDTH = 0.5
BATCH = 64
E2E_STEPS = 100
E2E_BATCHES = 5
METRIC = "grid-point steps/sec"
UNIT = "grid-pt*steps/s"
BYTES_PER_PT_PASS = 8  # FP32 state read + write per pass (algorithmic)


def V(x):
    return 0.05 * x ** 4 - x ** 2


def K(p):
    return 0.5 * p ** 2


def dV(x):
    return 0.2 * x ** 3 - 2.0 * x


def dK(p):
    return p


def initial_states(rng, batch, X, P):
    """Wigner functions of Gaussian wave packets psi ~ exp(-(x-x0)^2/(2w^2) + i p0 x)."""
    x0 = rng.uniform(-2.0, 2.0, size=batch)
    p0 = rng.uniform(-1.0, 1.0, size=batch)
    out = np.empty((batch, P.shape[0], X.shape[1]), dtype=np.float32)
    for b in range(batch):
        out[b] = (np.exp(-((X - x0[b]) ** 2) / WIDTH ** 2 - WIDTH ** 2 * (P - p0[b]) ** 2) / np.pi).astype(np.float32)
    return out


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(dist, x, device="cuda"):
    """The largest per-rank value (device-timed milliseconds) on every rank."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(units_per_rank, steps, world, el_ms):
    """Whole-job throughput of a weak-scaling run: every rank advanced
    units_per_rank units for `steps` steps; the job took el_ms (max over ranks)."""
    return units_per_rank * steps * world / (el_ms * 1e-3)


# ---------------------------------------------------------------------------
def measured_peak_gbs():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (read + write) per grid point of one column-pass launch, from an
# ncu capture of the persistent column pass (dram__bytes_read.sum +
# dram__bytes_write.sum of a 40-instance 1024 x 1024 launch: 175.5 + 137.9 MB,
# over its points); the line's roofline.traffic scales it to the points of one
# bench launch.
NCU_COL_DRAM_BYTES_PER_POINT = 7.47


def parity_check(sim, W0, steps=20):
    """Outside the timed region: restart the bench plan from the initial
    states, advance it `steps` steps and compare its first and last instance
    with the FP64 oracle (the checker, oracle/wigner_oracle.py).  Returns
    the largest relative L2 error of W and the largest error of an Ehrenfest
    observable relative to that observable's largest magnitude."""
    import torch

    from oracle.wigner_oracle import WignerOracle

    sim.t = 0.0
    sim.set_wignerfunctions(W0.cuda())
    W0n = sim.W.double().cpu().numpy()
    obs = sim.propagate(steps).cpu().numpy()
    torch.cuda.synchronize()
    W = sim.W.double().cpu().numpy()
    rel_l2, obs_rel = 0.0, 0.0
    insts = sorted({0, sim.batch - 1})
    for b in insts:
        o = WignerOracle(X_gridDIM=GRID, X_amplitude=AMP, P_gridDIM=GRID, P_amplitude=AMP, dt=DT, V=V, K=K,
                         diff_V=dV, diff_K=dK, fft_workers=os.cpu_count())
        o.cache_exponents()
        o.set_wignerfunction(W0n[b])
        o.propagate(steps)
        rel_l2 = max(rel_l2, float(np.linalg.norm(W[b] - o.W) / np.linalg.norm(o.W)))
        s = obs[:, b, 0]
        got = {"X_average": obs[:, b, 2] / s, "P_average_RHS": -obs[:, b, 3] / s, "P_average": obs[:, b, 5] / s,
               "X_average_RHS": obs[:, b, 6] / s, "hamiltonian_average": (obs[:, b, 4] + obs[:, b, 7]) / s}
        for k, g in got.items():
            r = np.asarray(getattr(o, k))
            obs_rel = max(obs_rel, float(np.abs(g - r).max() / np.abs(r).max()))
    return {"rel_l2": rel_l2, "max_obs_rel": obs_rel, "steps": steps, "instances": insts,
            "against": "FP64 oracle (numpy restatement of WignerMoyalFTTW1D.propagate)", "tol_rel_l2": 1e-5}


def uneven_parity(sim, steps=5):
    """Outside the timed region: the uneven batch (in the mode the autotuner
    picked) advances `steps` more steps from its current states; its smallest
    and largest instances are compared with the FP64 oracle (the checker,
    oracle/wigner_oracle.py) run from the same states."""
    import torch

    from oracle.wigner_oracle import WignerOracle

    sizes = [s["P_gridDIM"] * s["X_gridDIM"] for s in sim.specs]
    insts = sorted({int(np.argmin(sizes)), int(np.argmax(sizes))})
    W0 = [sim.W[i].double().cpu().numpy() for i in insts]
    t0 = sim.t
    sim.propagate(steps, use_graph=False)
    torch.cuda.synchronize()
    rel = 0.0
    for i, w0 in zip(insts, W0):
        s = sim.specs[i]
        o = WignerOracle(X_gridDIM=s["X_gridDIM"], X_amplitude=s["X_amplitude"], P_gridDIM=s["P_gridDIM"],
                         P_amplitude=s["P_amplitude"], dt=sim.dt, V=s["V"], K=s["K"], t=t0,
                         fft_workers=os.cpu_count())
        o.set_wignerfunction(w0)
        o.propagate(steps)
        W = sim.W[i].double().cpu().numpy()
        rel = max(rel, float(np.linalg.norm(W - o.W) / np.linalg.norm(o.W)))
    return {"rel_l2": rel, "steps": steps, "instances": insts,
            "grids": [[sim.specs[i]["P_gridDIM"], sim.specs[i]["X_gridDIM"]] for i in insts],
            "mode": sim.variant, "status": sim.status(),
            "against": "FP64 oracle from the batch's own states after the timed calls", "tol_rel_l2": 1e-5}


def fp64_256_parity(sim, kw, steps=5):
    """Outside the timed region: the FP64 256^2 batch advances `steps` more
    steps from its current states; its first and last instances are compared
    with the FP64 oracle run from the same states (tolerance 1e-10)."""
    import torch

    from oracle.wigner_oracle import WignerOracle

    insts = sorted({0, sim.batch - 1})
    W0 = [sim.W[b].cpu().numpy() for b in insts]
    t0 = sim.t
    sim.propagate(steps)
    torch.cuda.synchronize()
    rel = 0.0
    for b, w0 in zip(insts, W0):
        o = WignerOracle(X_gridDIM=kw["X_gridDIM"], X_amplitude=kw["X_amplitude"], P_gridDIM=kw["P_gridDIM"],
                         P_amplitude=kw["P_amplitude"], dt=kw["dt"], V=kw["V"], K=kw["K"], t=t0,
                         fft_workers=os.cpu_count())
        o.set_wignerfunction(w0)
        o.propagate(steps)
        rel = max(rel, float(np.linalg.norm(sim.W[b].cpu().numpy() - o.W) / np.linalg.norm(o.W)))
    return {"rel_l2": rel, "steps": steps, "instances": insts,
            "against": "FP64 oracle from the batch's own states after the timed calls", "tol_rel_l2": 1e-10}


def vn_1024_parity(q, steps=5):
    """Outside the timed region: the complex64 von Neumann propagator of the
    vn_1024 workload (double well 0.05 x^4 - x^2, K = p^2/2) advances `steps`
    more steps from its current density matrix; compared with the FP64 density-
    matrix oracle (oracle/rho_oracle.py) run from the same matrix."""
    from oracle.rho_oracle import RhoOracle

    R0 = q.rho.get().astype(np.complex128)
    t0 = q.t
    R = q.propagate(steps).get()
    o = RhoOracle(X_gridDIM=1024, X_amplitude=10.0, dt=0.005, t=t0, V=lambda x: 0.05 * x ** 4 - x ** 2,
                  K=lambda p: 0.5 * p * p)
    o.set_rho(R0)
    o.propagate(steps)
    return {"rel_l2": float(np.linalg.norm(R - o.rho) / np.linalg.norm(o.rho)), "steps": steps,
            "against": "FP64 density-matrix oracle from the propagator's own state after the timed calls",
            "tol_rel_l2": 1e-5}


def bloch_512_parity(bb, setup, Ds, As, steps=5):
    """Outside the timed region: the Morse Bloch batch advances `steps` more
    imaginary-time steps from its current states; its first and last instances
    are compared with the FP64 oracle's CUDA-convention Bloch step
    (wigner_bloch_cuda_1d.py:229-254) run from the same states."""
    import torch

    from oracle.wigner_oracle import WignerOracle

    insts = sorted({0, bb.n - 1})
    W0 = [bb.W[i].double().cpu().numpy() for i in insts]
    bb.run(steps)
    torch.cuda.synchronize()
    rel = 0.0
    for i, w0 in zip(insts, W0):
        o = WignerOracle(X_gridDIM=setup.G, X_amplitude=setup.XA, P_gridDIM=setup.G, P_amplitude=setup.PA,
                         dt=setup.dbeta, V=setup.V(Ds[i], As[i]), K=lambda p: 0.5 * p * p, fft_workers=os.cpu_count())
        o.setup_bloch_cuda()
        o.set_wignerfunction(w0)
        for _ in range(steps):
            o.bloch_single_step(setup.dbeta)
        rel = max(rel, float(np.linalg.norm(bb.W[i].double().cpu().numpy() - o.W) / np.linalg.norm(o.W)))
    return {"rel_l2": rel, "steps": steps, "instances": insts,
            "against": "FP64 oracle (CUDA-convention Bloch step) from the batch's own states after the timed calls",
            "tol_rel_l2": 1e-5}


WORKLOAD_CHECKS = {"batch_uneven": uneven_parity, "moyal_fp64_256": fp64_256_parity, "vn_1024": vn_1024_parity,
                   "bloch_512": bloch_512_parity}


# The other configurations (fastwigner_b200/benchmarks.py), measured after the
# headline on the same GPU so that every run records them: config 1 (FP64 Moyal
# 256^2), config 2b (von Neumann complex64 1024^2), config 3 (Bloch 512^2 Morse
# batch), config 4 (uneven persistent batch) and config 5 (strong field with
# collisions).  Each entry is that workload's own line, trimmed.
OTHER_WORKLOADS = ("moyal_fp64_256", "vn_1024", "bloch_512", "batch_uneven", "strong_field", "fno_predict_512")


def other_workloads():
    from fastwigner_b200 import benchmarks

    out = {}
    for name in OTHER_WORKLOADS:
        try:
            kw = {"check": WORKLOAD_CHECKS[name]} if name in WORKLOAD_CHECKS else {}
            line = benchmarks.run(name, **kw)
            out[name] = {"value": line["value"], "unit": line["unit"], "ms_per_step": line["ms_per_step"],
                         "dtype": line["dtype"], "roofline_frac": line["roofline"]["frac"],
                         "algorithmic_bytes_per_unit": line["roofline"]["algorithmic_bytes_per_unit"],
                         "clocks_sm_mhz": line["clocks"].get("sm_mhz"), "config": line["config"]}
            if "parity" in line:
                out[name]["parity"] = line["parity"]
        except Exception as e:  # a failing side workload must not cost the headline line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


# ---------------------------------------------------------------------------
def cpu_reference_rate(target_s, steps=None, grid=GRID, workers=None):
    """Time the FP64 oracle port (the reference algorithm; FFTs on `workers`
    threads, all host cores by default) on one instance; returns
    (pt-steps/s, steps run, seconds, threads)."""
    from oracle.wigner_oracle import WignerOracle

    cores = workers or os.cpu_count() or 1
    o = WignerOracle(X_gridDIM=grid, X_amplitude=AMP, P_gridDIM=grid, P_amplitude=AMP, dt=DT,
                     V=V, K=K, diff_V=dV, diff_K=dK, fft_workers=cores)
    o.cache_exponents()
    rng = np.random.default_rng(12345)
    o.set_wignerfunction(initial_states(rng, 1, o.X, o.P)[0].astype(np.float64))
    o.propagate(2)  # warm-up (plans, page faults)
    if steps is None:
        t0 = time.perf_counter()
        o.propagate(3)
        per = (time.perf_counter() - t0) / 3
        steps = max(3, int(target_s / per))
    t0 = time.perf_counter()
    o.propagate(steps)
    el = time.perf_counter() - t0
    return grid * grid * steps / el, steps, el, cores


REF_SAMPLE_INSTANCES = 8  # instances of the batch the reference arm advances per bench step


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    from oracle.wigner_oracle import WignerOracle

    n = min(REF_SAMPLE_INSTANCES, args.batch)
    rng = np.random.default_rng(12345)
    inst = []
    for _ in range(n):
        o = WignerOracle(X_gridDIM=GRID, X_amplitude=AMP, P_gridDIM=GRID, P_amplitude=AMP, dt=DT,
                         V=V, K=K, diff_V=dV, diff_K=dK, fft_workers=cores)
        o.cache_exponents()
        o.set_wignerfunction(initial_states(rng, 1, o.X, o.P)[0].astype(np.float64))
        inst.append(o)

    def step():  # one time step of the sampled instances
        for o in inst:
            o.propagate(1)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    value = GRID * GRID * n * args.steps / el
    sample = (f"{n} instances of the {GRID}x{GRID} workload per step, {args.steps} FP64 steps, "
              f"scipy.fft workers={cores}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"moyal_double_well_{GRID}x{GRID}_batch{args.batch}", "grid": [GRID, GRID],
                   "batch_per_gpu": args.batch, "dt": DT, "potential": "0.05 x^4 - x^2", "amplitudes": [AMP, AMP],
                   "sample": f"{n} of the {args.batch} instances per step (the metric is per grid point)",
                   "implementation": "FP64 numpy restatement of WignerMoyalFTTW1D"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from fastwigner_b200 import _lib
    from fastwigner_b200.batch import WignerMoyalBatch
    from fastwigner_b200.benchmarks import ClockSampler

    B = args.batch
    sim = WignerMoyalBatch(batch=B, X_gridDIM=GRID, X_amplitude=AMP, P_gridDIM=GRID, P_amplitude=AMP, dt=DT,
                           V=V, K=K, diff_V=dV, diff_K=dK, precision="float32")
    rng = np.random.default_rng(1000 + rank)
    W0 = initial_states(rng, B, sim.X, sim.P)
    W0_pinned = torch.from_numpy(W0).pin_memory()
    sim.set_wignerfunctions(W0_pinned.cuda())
    lib = _lib.load()
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up
    obs = torch.empty((max(args.steps, E2E_STEPS), B, 8), dtype=torch.float64, device="cuda")
    sim.propagate(args.warmup, obs=obs[: args.warmup])
    torch.cuda.synchronize()

    # ---- timed region: K steps of all instances, inputs resident in HBM -------
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    n0 = lib.fw_launch_count()
    with ClockSampler(local) as clk:
        start.record(stream)
        sim.propagate(args.steps, obs=obs[: args.steps])
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = lib.fw_launch_count() - n0
    el_ms = max_over_ranks(dist, start.elapsed_time(end))
    pts = GRID * GRID * B
    value = job_value(pts, args.steps, world, el_ms)
    # sanity: the states stay normalised and finite
    o = obs[args.steps - 1].cpu().numpy()
    finite = bool(np.isfinite(o).all())

    # ---- per-kernel timing (CUDA events between launches on the same stream) ---
    _, ms, kind = sim.propagate_timed(min(50, args.steps))
    col = ms[kind == 0][1:]  # skip the opening half-step launch
    row = ms[kind == 1]
    col_ms, row_ms = float(np.mean(col)), float(np.mean(row))
    dom_kind, dom_ms = ("column pass (FFT_p, exp(V_k) x exp(V_k+1) with observables from the mid-point spectrum, iFFT_p)", col_ms) \
        if col.sum() >= row.sum() else ("row pass (FFT_x, exp(K), iFFT_x)", row_ms)
    peak, peak_kind = measured_peak_gbs()
    alg_bytes = BYTES_PER_PT_PASS * pts
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": NCU_COL_DRAM_BYTES_PER_POINT * pts,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per point of a 40-instance "
                                  "column-pass launch (captured separately), times the points of one launch",
                "kernel": dom_kind, "kernel_ms": dom_ms, "col_ms": col_ms, "row_ms": row_ms,
                "algorithmic_bytes_per_launch": alg_bytes, "peak_kind": f"{peak_kind} hbm_gbs",
                "frac_of_nominal_8000_gbs": achieved / 8000.0}

    # ---- end-to-end through the public API: pinned host states in, results out --
    # E2E_BATCHES host batches stream through propagate_host_batches: each is
    # copied in from pinned memory, normalised, propagated E2E_STEPS steps and
    # copied back with its observables, the copies overlapping the neighbouring
    # batches' propagation (two alternating host output buffers); only the
    # first copy-in and the last copy-out have no neighbour to hide behind.
    # The same five batches whatever --steps is (about 0.25 s of work).
    e2e_calls = E2E_BATCHES
    host_out = [torch.empty((B, GRID, GRID), dtype=torch.float32).pin_memory() for _ in range(2)]
    obs_host = [torch.empty((E2E_STEPS, B, 8), dtype=torch.float64).pin_memory() for _ in range(2)]
    # untimed warm-up of the same call (allocates its second device state buffer)
    sim.propagate_host_batches([W0_pinned] * 2, 1, out=host_out,
                               obs_out=[o[:1] for o in obs_host])
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.propagate_host_batches([W0_pinned] * e2e_calls, E2E_STEPS,
                               out=[host_out[i & 1] for i in range(e2e_calls)],
                               obs_out=[obs_host[i & 1] for i in range(e2e_calls)])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(dist, e0.elapsed_time(e1))
    e2e_value = job_value(pts, E2E_STEPS * e2e_calls, world, e2e_ms)
    e2e_finite = bool(np.isfinite(obs_host[(e2e_calls - 1) & 1].numpy()).all())
    h2d = W0_pinned.numel() * 4 / E2E_STEPS
    d2h = (host_out[0].numel() * 4 + obs_host[0].numel() * 8) / E2E_STEPS

    parity = parity_check(sim, W0_pinned) if rank == 0 else None
    others = other_workloads() if rank == 0 and world == 1 and not args.no_workloads else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, csteps, cel, cores = cpu_reference_rate(args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"1 instance of the {GRID}x{GRID} workload, {csteps} FP64 steps in {cel:.1f} s "
                         f"(numpy restatement of WignerMoyalFTTW1D, scipy.fft workers={cores})"}
        r1, s1, e1_, _ = cpu_reference_rate(args.cpu_seconds / 3, workers=1)
        cpu["single_thread"] = {"value": r1, "unit": UNIT, "cores": 1,
                                "sample": f"the same instance, {s1} FP64 steps in {e1_:.1f} s, scipy.fft workers=1"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"moyal_double_well_{GRID}x{GRID}_batch{B}", "grid": [GRID, GRID],
                       "batch_per_gpu": B, "dt": DT, "potential": "0.05 x^4 - x^2", "amplitudes": [AMP, AMP],
                       "state_bytes_per_gpu": pts * 4, "l2_policy": "inputs larger than L2 (256 MiB states)",
                       "passes_per_step": 2, "observables_per_step": 8, "finite": finite,
                       "e2e_call": f"propagate_host_batches: {e2e_calls} pinned host batches, each copied in, "
                                   f"normalised, propagated {E2E_STEPS} steps, states and observables copied "
                                   f"back to pinned host (copies overlap the neighbouring batches)",
                       "e2e_finite": e2e_finite},
            "roofline": roofline,
            "parity": parity,
            "workloads": others,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="skip the other configurations' figures")
    ap.add_argument("--workload", default="moyal_1024",
                    help="moyal_1024 (the default line) or one of fastwigner_b200.benchmarks.WORKLOADS")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "moyal_1024":
        from fastwigner_b200 import benchmarks

        if args.workload not in benchmarks.WORKLOADS:
            ap.error(f"unknown workload {args.workload}")
        kw = {"check": WORKLOAD_CHECKS[args.workload]} if args.workload in WORKLOAD_CHECKS else {}
        print(json.dumps(benchmarks.run(args.workload, **kw)), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
