"""Throughput of the propagators on the synthetic workloads other than the
headline 1024^2 Moyal batch (which ``bench.py`` measures by default).

Each workload prints one JSON line in the format of ``bench.py``'s line:
grid-point (or matrix-element) steps per second, CUDA-event timed on the
launching stream after warm-up, with the algorithmic HBM bytes per unit and
the resulting fraction of the measured copy bandwidth.  Sizes, parameters and
seeds follow the workloads the propagators are specified on:

* ``moyal_fp64_256`` -- Moyal, FP64, 256^2, X/P amplitudes 8/7, dt 0.01,
  V = x^2/2, K = p^2/2, W0 = exp(-(x-1)^2 - (p-0.5)^2)/pi, 4 observables per
  step.  One instance is L2-resident (512 KiB); the line also times a batch of
  512 copies (256 MiB) so that every pass streams from HBM.
* ``vn_1024`` -- von Neumann rho(x, x'), complex64, 1024^2, double well
  V = 0.05 x^4 - x^2, amplitude 10, dt 0.005, rho = psi psi* of a Gaussian
  packet (x0 ~ U(-2, 2), p0 ~ U(-1, 1), width 0.5).  8 MiB: L2-resident.
* ``bloch_512`` -- imaginary-time Bloch steps, FP32, 512^2, Morse
  V = D (1 - exp(-a (x - x_e)))^2 with D ~ U(2, 10), a ~ U(0.5, 1.5),
  dbeta = 1e-3, 16 instances with their own exponent tables.
* ``batch_uneven`` -- 256 independent FP32 Moyal instances, grids drawn per
  axis from {128, 256, 512, 1024}, double wells a x^4 - b x^2 with
  a ~ U(0.02, 0.1), b ~ U(0.5, 2), amplitude 10, dt 0.005, one persistent
  cooperative launch per call replayed as a CUDA graph (launch shape from the
  autotuner).
* ``strong_field`` -- velocity-gauge laser-driven soft-core atom with
  random-collision dephasing: V0 = -1/sqrt(x^2 + 1), E(t) = E0 sin^2(pi t/T)
  sin(w t), E0 ~ U(0.01, 0.1), w = 0.057, T = 8 cycles, x: 2048 points
  (amplitude 200), p: 1024 (amplitude 5), dt 0.05, gamma ~ U(1e-4, 1e-2),
  FP32 with the field integral in FP64.  8 MiB per state: L2-resident.
"""
from __future__ import annotations

import json
import math

import numpy as np
import torch

WORKLOADS = ("moyal_fp64_256", "vn_1024", "bloch_512", "batch_uneven", "strong_field")


def _peak():
    from pathlib import Path

    try:
        d = json.loads((Path(__file__).resolve().parent.parent / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured hbm_gbs"
    except Exception:
        return 6650.0, "fallback hbm_gbs"


def _timed(fn, warm=1):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e)


def _line(name, value, unit, steps, ms, dtype, bytes_per_unit, config, extra=None):
    peak, kind = _peak()
    gbs = value * bytes_per_unit / 1e9
    line = {"workload": name, "metric": "grid-point steps/sec" if "pt" in unit else "matrix-element steps/sec",
            "value": value, "unit": unit, "n_gpus": 1, "steps": steps, "ms_per_step": ms / steps,
            "higher_is_better": True, "dtype": dtype, "data": "synthetic", "config": config,
            "roofline": {"bound": "hbm", "algorithmic_bytes_per_unit": bytes_per_unit, "achieved": gbs,
                         "peak": peak, "unit": "GB/s", "frac": gbs / peak, "peak_kind": kind}}
    if extra:
        line.update(extra)
    return line


# ---------------------------------------------------------------------------
def moyal_fp64_256(steps=1000, big_batch=512):
    from .batch import WignerMoyalBatch

    kw = dict(X_gridDIM=256, X_amplitude=8.0, P_gridDIM=256, P_amplitude=7.0, dt=0.01,
              V=lambda x: 0.5 * x * x, K=lambda p: 0.5 * p * p, diff_V=lambda x: x, diff_K=lambda p: p,
              precision="float64")
    res = {}
    for B in (1, big_batch):
        sim = WignerMoyalBatch(batch=B, **kw)
        W0 = np.exp(-((sim.X - 1.0) ** 2) - (sim.P - 0.5) ** 2) / np.pi
        sim.set_wignerfunctions(torch.from_numpy(np.broadcast_to(W0, (B, 256, 256)).copy()).cuda())
        obs = torch.empty((steps, B, 8), dtype=torch.float64, device="cuda")
        ms = _timed(lambda: sim.propagate(steps, obs=obs))
        res[B] = (256 * 256 * B * steps / (ms * 1e-3), ms)
        del sim
    v, ms = res[big_batch]
    return _line("moyal_fp64_256", v, "grid-pt*steps/s", steps, ms, "f64", 32,
                 {"grid": [256, 256], "amplitudes": [8.0, 7.0], "dt": 0.01, "batch": big_batch,
                  "passes_per_step": 2, "l2_policy": f"batch of {big_batch} copies (256 MiB) streams from HBM"},
                 {"single_instance": {"value": res[1][0], "ms_per_step": res[1][1] / steps,
                                      "note": "512 KiB state, L2-resident"}})


def vn_1024(steps=400):
    from .rho import RhoVNeumannCUDA1D

    q = RhoVNeumannCUDA1D(X_gridDIM=1024, X_amplitude=10.0, dt=0.005, t=0.0, K="0.5 * P * P",
                          V="0.05 * X * X * X * X - X * X", diff_K="P", diff_V="0.2 * X * X * X - 2.0 * X",
                          precision="float32")
    rng = np.random.default_rng(7)
    x0, p0 = rng.uniform(-2, 2), rng.uniform(-1, 1)
    x = q.X.reshape(-1)
    psi = np.exp(-((x - x0) ** 2) / (2 * 0.5 ** 2) + 1j * p0 * x)
    q.set_rho(psi[:, None] * psi.conj()[None, :])
    ms = _timed(lambda: q.propagate(steps))
    n = 1024 * 1024
    return _line("vn_1024", n * steps / (ms * 1e-3), "matrix-el*steps/s", steps, ms, "c64", 32,
                 {"grid": [1024, 1024], "amplitude": 10.0, "dt": 0.005, "passes_per_step": 2,
                  "observables_per_step": 5, "l2_policy": "8 MiB state, L2-resident (effective figure)"})


def bloch_512(steps=2000, n=16):
    from .fno import BlochBatch, MorseBlochSetup

    rng = np.random.default_rng(3)
    Ds, As = rng.uniform(2, 10, n), rng.uniform(0.5, 1.5, n)
    setup = MorseBlochSetup()
    bb = BlochBatch(setup, Ds, As).set_uniform()
    ms = _timed(lambda: bb.run(steps))
    pts = setup.G * setup.G * n
    return _line("bloch_512", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 16,
                 {"grid": [setup.G, setup.G], "instances": n, "dbeta": setup.dbeta, "passes_per_step": 2,
                  "state_bytes": pts * 4, "l2_policy": "16 MiB of states, mostly L2-resident"})


def batch_uneven(steps=2000, n=256):
    from .batch import WignerMoyalUnevenBatch

    rng = np.random.default_rng(11)
    sizes = (128, 256, 512, 1024)
    specs = []
    for _ in range(n):
        a, b = rng.uniform(0.02, 0.1), rng.uniform(0.5, 2.0)
        specs.append(dict(P_gridDIM=int(rng.choice(sizes)), X_gridDIM=int(rng.choice(sizes)), X_amplitude=10.0,
                          P_amplitude=10.0, V=(lambda x, a=a, b=b: a * x ** 4 - b * x ** 2),
                          K=(lambda p: 0.5 * p ** 2)))
    sim = WignerMoyalUnevenBatch(specs, dt=0.005)
    states = []
    for s in sim.specs:  # the batch keeps its own copies, with the grids filled in
        x0, p0 = rng.uniform(-2, 2), rng.uniform(-1, 1)
        states.append(np.exp(-((s["X"] - x0) ** 2) / 0.25 - 0.25 * (s["P"] - p0) ** 2))
    sim.set_wignerfunctions(states)
    obs = torch.empty((steps, n, 2), dtype=torch.float64, device="cuda")
    ms = _timed(lambda: sim.propagate(steps, use_graph=True, obs=obs))
    pts = sum(s["P_gridDIM"] * s["X_gridDIM"] for s in specs)
    return _line("batch_uneven", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 16,
                 {"instances": n, "grids_per_axis": list(sizes), "total_points": pts, "state_bytes": pts * 4,
                  "variant": sim.variant, "graph": True, "passes_per_step": 2,
                  "l2_policy": f"{pts * 4 / 2**20:.0f} MiB of states, above L2"},
                 {"status": sim.status()})


def strong_field(steps=500):
    from .strong_field import StrongFieldWigner

    rng = np.random.default_rng(5)
    E0, w, gamma = rng.uniform(0.01, 0.1), 0.057, rng.uniform(1e-4, 1e-2)
    T = 8 * 2 * math.pi / w

    def E(_, t):  # vectorised: the FP64 field integral evaluates it at quadrature nodes
        return E0 * np.sin(np.pi * t / T) ** 2 * np.sin(w * t)

    q = StrongFieldWigner(X_gridDIM=2048, X_amplitude=200.0, P_gridDIM=1024, P_amplitude=5.0, dt=0.05, t=0.0,
                          V=lambda _, x: -1.0 / np.sqrt(x * x + 1.0), diff_V=lambda _, x: x / (x * x + 1.0) ** 1.5,
                          gauge="velocity", E=E, gamma=gamma, kT=0.1, dbeta=0.01, precision="float32")
    q.set_wignerfunction(q.gibbs_state)
    ms = _timed(lambda: q.propagate(steps))
    pts = 2048 * 1024
    return _line("strong_field", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 32,
                 {"grid_x": 2048, "grid_p": 1024, "amplitudes": [200.0, 5.0], "dt": 0.05, "E0": E0, "omega": w,
                  "cycles": 8, "gamma": gamma, "kT": 0.1, "dbeta": 0.01, "gauge": "velocity", "passes_per_step": 3,
                  "l2_policy": "8 MiB state, L2-resident (effective figure)"})


def run(name, **kw):
    return globals()[name](**kw)
