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
  a ~ U(0.02, 0.1), b ~ U(0.5, 2), amplitude 10, dt 0.005, replayed as a
  CUDA graph; the autotuner picks between the launch shapes of the persistent
  cooperative kernel (one launch per call) and the grouped mode (one plan per
  grid shape, the groups one after another in one graph).
* ``strong_field`` -- velocity-gauge laser-driven soft-core atom with
  random-collision dephasing: V0 = -1/sqrt(x^2 + 1), E(t) = E0 sin^2(pi t/T)
  sin(w t), E0 ~ U(0.01, 0.1), w = 0.057, T = 8 cycles, x: 2048 points
  (amplitude 200), p: 1024 (amplitude 5), dt 0.05, gamma ~ U(1e-4, 1e-2),
  FP32 with the field integral in FP64.  8 MiB per state: L2-resident.
"""
from __future__ import annotations

import json
import math
import os
import statistics
import subprocess
import threading

import numpy as np
import torch

WORKLOADS = ("moyal_fp64_256", "vn_1024", "bloch_512", "batch_uneven", "strong_field", "strong_field_frames",
             "rho_to_wigner_1024", "moyal_absorbing_1024", "fno_predict_512")

# NVML clock-event reason bits (nvmlClocksEventReason*): reported when active.
_REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}


class ClockSampler:
    """SM clock and clock-event reasons sampled while a timed region runs.

    Used as a context manager around the region: a thread reads NVML every
    `interval` seconds from entry to exit (kernels run asynchronously, so the
    host polls while the enqueued work executes, and even a region of a few
    milliseconds gets samples).  Falls back to `nvidia-smi -lms 200` when NVML
    is unavailable.  Only reads the GPU's state."""

    SMI_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=None, interval=0.01):
        self.device_index = torch.cuda.current_device() if device_index is None else device_index
        self.interval = interval
        self.sm, self.mx, self.reasons, self.source = [], [], set(), "unsampled"
        self._stop = threading.Event()
        self._thread = self._proc = self._nvml = self._handle = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        self._nvml = pynvml
        props = torch.cuda.get_device_properties(self.device_index)
        try:
            u = str(props.uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            pass
        bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
        return pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _sample_nvml(self):
        nv, h = self._nvml, self._handle
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.sm.append(float(sm))
        self.mx.append(float(mx))
        self.reasons.update(n for n, b in _REASON_BITS.items() if bits & b)

    def _loop(self):
        while True:
            try:
                self._sample_nvml()
            except Exception:
                return
            if self._stop.wait(self.interval):
                return

    def __enter__(self):
        try:
            self._handle = self._nvml_handle()
            self._sample_nvml()
            self.sm, self.mx, self.reasons = [], [], set()  # the entry sample only checks the handle
            self.source = "nvml"
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
        except Exception:
            self._handle = None
            try:
                idx = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[self.device_index].strip() or str(
                    self.device_index)
            except IndexError:
                idx = str(self.device_index)
            try:
                self._proc = subprocess.Popen(
                    ["nvidia-smi", "-i", idx, f"--query-gpu={self.SMI_QUERY}", "--format=csv,noheader,nounits",
                     "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi"
            except OSError:
                self._proc = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self._nvml is not None:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass
        if self._proc is not None:
            self._proc.terminate()
            try:
                out, _ = self._proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
                out, _ = self._proc.communicate()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for ln in out.splitlines():
                f = [c.strip() for c in ln.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm, mx = float(f[1]), float(f[2])
                except ValueError:
                    continue
                self.sm.append(sm)
                self.mx.append(mx)
                self.reasons.update(n for n, v in zip(names, f[5:9]) if v.lower().startswith("active"))
        return False

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": max(self.mx), "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": self.source}


def _peak():
    from pathlib import Path

    try:
        d = json.loads((Path(__file__).resolve().parent.parent / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured hbm_gbs"
    except Exception:
        return 6650.0, "fallback hbm_gbs"


_last_clocks = {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}


def _timed(fn, warm=2, reps=3):
    """Median device time (ms) of `reps` calls of fn after `warm` untimed calls;
    the SM clocks seen during the timed calls go into the workload's line."""
    global _last_clocks
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    out = []
    with ClockSampler() as clk:
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            out.append(s.elapsed_time(e))
    _last_clocks = clk.summary()
    return float(np.median(out))


def _line(name, value, unit, steps, ms, dtype, bytes_per_unit, config, extra=None):
    peak, kind = _peak()
    gbs = value * bytes_per_unit / 1e9
    line = {"workload": name, "metric": "grid-point steps/sec" if "pt" in unit else "matrix-element steps/sec",
            "value": value, "unit": unit, "n_gpus": 1, "steps": steps, "ms_per_step": ms / steps,
            "higher_is_better": True, "dtype": dtype, "data": "synthetic", "config": config,
            "roofline": {"bound": "hbm", "algorithmic_bytes_per_unit": bytes_per_unit, "achieved": gbs,
                         "peak": peak, "unit": "GB/s", "frac": gbs / peak, "peak_kind": kind},
            "clocks": _last_clocks}
    if extra:
        line.update(extra)
    return line


# ---------------------------------------------------------------------------
def moyal_fp64_256(steps=1000, big_batch=512, check=None):
    """``check``: optional callable given the big batch after its timed calls
    and the constructor keywords (outside the timing); its result goes into
    the line as ``parity``."""
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
        if B == big_batch and check is not None:
            res["parity"] = check(sim, kw)
        del sim
    v, ms = res[big_batch]
    extra = {"single_instance": {"value": res[1][0], "ms_per_step": res[1][1] / steps,
                                 "note": "512 KiB state, L2-resident"}}
    if "parity" in res:
        extra["parity"] = res["parity"]
    return _line("moyal_fp64_256", v, "grid-pt*steps/s", steps, ms, "f64", 32,
                 {"grid": [256, 256], "amplitudes": [8.0, 7.0], "dt": 0.01, "batch": big_batch,
                  "passes_per_step": 2, "l2_policy": f"batch of {big_batch} copies (256 MiB) streams from HBM"},
                 extra)


def vn_1024(steps=400, check=None):
    """``check``: optional callable given the propagator after its timed calls
    (outside the timing); its result goes into the line as ``parity``."""
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
                  "observables_per_step": 5, "l2_policy": "8 MiB state, L2-resident (effective figure)"},
                 {"parity": check(q)} if check is not None else None)


def bloch_512(steps=2000, n=16, check=None):
    """``check``: optional callable given the batch, the setup and the Morse
    parameters after the timed calls (outside the timing); its result goes
    into the line as ``parity``."""
    from .fno import BlochBatch, MorseBlochSetup

    rng = np.random.default_rng(3)
    Ds, As = rng.uniform(2, 10, n), rng.uniform(0.5, 1.5, n)
    setup = MorseBlochSetup()
    bb = BlochBatch(setup, Ds, As).set_uniform()
    ms = _timed(lambda: bb.run(steps))
    pts = setup.G * setup.G * n
    return _line("bloch_512", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 16,
                 {"grid": [setup.G, setup.G], "instances": n, "dbeta": setup.dbeta, "passes_per_step": 2,
                  "state_bytes": pts * 4, "l2_policy": "16 MiB of states, mostly L2-resident"},
                 {"parity": check(bb, setup, Ds, As)} if check is not None else None)


def fno_predict_512(n=16):
    """Inference of the Bloch surrogate (4 Fourier layers, width 32, 16 x 16
    modes, 128-wide fused projection; random weights: timing only) for n Morse
    instances on the 512^2 grid, harmonic baseline and normalisation included.
    Algorithmic bytes per grid point: the 32-channel activations read or
    written 5 times per layer (forward x-DFT read, inverse x-DFT write, channel
    map reads of the input and of the inverse DFT, its write) x 4 layers, plus
    the lift's write and the projection's read: 22 x 128 B = 2816 B."""
    from .fno import BlochSurrogate, FNO2d, MorseBlochSetup

    setup = MorseBlochSetup()
    net = FNO2d(n_params=3, width=32, modes=(16, 16), layers=4, proj=128, seed=0)
    sur = BlochSurrogate(setup, net)
    rng = np.random.default_rng(5)
    Ds, As = rng.uniform(2, 10, n), rng.uniform(0.5, 1.5, n)
    ms = _timed(lambda: sur.predict(Ds, As, 4.0))
    pts = setup.G * setup.G * n
    line = _line("fno_predict_512", pts / (ms * 1e-3), "grid-pt/s", 1, ms, "f32", 2816,
                 {"grid": [setup.G, setup.G], "instances": n, "layers": 4, "width": 32, "modes": [16, 16],
                  "projection": 128, "gemm": "tcgen05 TF32, three-way split", "weights": "random (timing only)"})
    line["metric"] = "grid points per second (surrogate inference)"
    return line


def batch_uneven(steps=2000, n=256, check=None):
    """``check``: optional callable given the batch after the timed calls
    (outside the timing); what it returns goes into the line as ``parity``."""
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
    extra = {"status": sim.status()}
    if check is not None:
        extra["parity"] = check(sim)
    return _line("batch_uneven", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 16,
                 {"instances": n, "grids_per_axis": list(sizes), "total_points": pts, "state_bytes": pts * 4,
                  "variant": sim.variant, "variants": {"persistent": list(range(sim.GROUPED)), "grouped": sim.GROUPED},
                  "autotune_ms_per_step": getattr(sim, "autotune_ms", None), "graph": True, "passes_per_step": 2,
                  "l2_policy": f"{pts * 4 / 2**20:.0f} MiB of states, above L2"},
                 extra)


def _strong_field_sim():
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
    return q, E0, w, gamma


def strong_field(steps=500):
    q, E0, w, gamma = _strong_field_sim()
    ms = _timed(lambda: q.propagate(steps))
    pts = 2048 * 1024
    return _line("strong_field", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 32,
                 {"grid_x": 2048, "grid_p": 1024, "amplitudes": [200.0, 5.0], "dt": 0.05, "E0": E0, "omega": w,
                  "cycles": 8, "gamma": gamma, "kT": 0.1, "dbeta": 0.01, "gauge": "velocity", "passes_per_step": 3,
                  "l2_policy": "8 MiB state, L2-resident (effective figure)"})


def strong_field_frames(steps=500, every=20):
    """strong_field with the Wigner function recorded every `every` steps
    through a FrameRecorder (propagate(steps, frames=..., frame_every=...):
    device snapshot on the compute stream, pinned-host copy on a side stream,
    4-slot ring, no wait between frames), all frames drained to host arrays
    inside the timed region; the plain run is timed beside it."""
    from .results import FrameRecorder

    q = _strong_field_sim()[0]
    rec = FrameRecorder(depth=4)

    def go():
        q.propagate(steps, frames=rec, frame_every=every)
        return rec.take()

    ms = _timed(go)
    plain = _timed(lambda: q.propagate(steps))
    pts = 2048 * 1024
    nf = steps // every
    return _line("strong_field_frames", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 32,
                 {"grid_x": 2048, "grid_p": 1024, "frames": nf, "frame_every": every,
                  "frame_bytes": pts * 4, "ring_depth": 4},
                 {"plain_ms_per_step": plain / steps, "frame_overhead": ms / plain - 1.0})


def rho_to_wigner_1024(reps=50):
    """The rho -> W transform (three shear passes, the sign-flipped FFT, the
    normalisation sum and scale) of the vn_1024 state, repeated."""
    from .rho import RhoVNeumannCUDA1D

    q = RhoVNeumannCUDA1D(X_gridDIM=1024, X_amplitude=10.0, dt=0.005, t=0.0, K="0.5 * P * P",
                          V="0.05 * X * X * X * X - X * X", precision="float32")
    rng = np.random.default_rng(7)
    x0, p0 = rng.uniform(-2, 2), rng.uniform(-1, 1)
    x = q.X.reshape(-1)
    psi = np.exp(-((x - x0) ** 2) / (2 * 0.5 ** 2) + 1j * p0 * x)
    q.set_rho(psi[:, None] * psi.conj()[None, :])
    q.propagate(20)

    def go():
        for _ in range(reps):
            q.get_wignerfunction()

    ms = _timed(go)
    n = 1024 * 1024
    # copy (16) + 3 shear passes (48) + sign / FFT pass (16) + sum (8) + scale (16) + clone (16)
    return _line("rho_to_wigner_1024", n * reps / (ms * 1e-3), "matrix-el/s", reps, ms, "c64", 120,
                 {"grid": [1024, 1024], "transforms": reps, "passes": 6,
                  "note": "one host read of the complex normalisation sum per transform",
                  "l2_policy": "8 MiB matrix, L2-resident (effective figure)"},
                 {"metric": "matrix elements transformed/sec", "ms_per_transform": ms / reps})


def moyal_absorbing_1024(steps=400):
    """WignerMoyalCUDA1D, FP32 1024^2 double well with the reference's x-p absorbing
    mask (wigner_moyal_cuda_1d.py:39-44): the mask sits between the closing and
    opening exp(V) half-steps, so the column pass runs its unfused form."""
    from .wigner_cuda import WignerMoyalCUDA1D

    q = WignerMoyalCUDA1D(X_gridDIM=1024, X_amplitude=10.0, P_gridDIM=1024, P_amplitude=10.0, dt=0.005, t=0.0,
                          K="0.5 * P * P", V="0.05 * X * X * X * X - X * X", diff_K="P",
                          diff_V="0.2 * X * X * X - 2.0 * X", precision="float32",
                          abs_boundary_x_p="pow(abs(sin(0.5 * M_PI * (X + X_amplitude) / X_amplitude)), dt * 0.5)")
    q.set_wignerfunction("exp(-(X - 1.0) * (X - 1.0) - 2.0 * P * P)")
    ms = _timed(lambda: q.propagate(steps))
    pts = 1024 * 1024
    return _line("moyal_absorbing_1024", pts * steps / (ms * 1e-3), "grid-pt*steps/s", steps, ms, "f32", 20,
                 {"grid": [1024, 1024], "dt": 0.005, "boundary": "abs_boundary_x_p = |sin(pi (X + A) / 2A)|^(dt/2)",
                  "passes_per_step": 2, "column_pass": "unfused (two transform pairs around the mask)",
                  "l2_policy": "4 MiB state, L2-resident (effective figure)"})


def run(name, **kw):
    return globals()[name](**kw)
