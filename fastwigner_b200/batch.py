"""Many independent Wigner functions on one grid, advanced together.

``WignerMoyalBatch`` runs B instances of the Moyal (or Bloch) split-operator
step in the same launches: every column/row pass covers all instances
(grid.y = instance), so a batch whose states exceed the 126 MB L2 streams
from HBM at the pass kernels' bandwidth.  Instances share one set of phase
tables (same Hamiltonian, different initial states -- e.g. random wave
packets) or carry their own (``V``/``K`` given as lists, one per instance).

The algorithm and conventions are WignerMoyalFTTW1D's
(wigner_moyal_fftw_1d.py:101-481): exponents at the incremented time,
renormalisation after every step, Ehrenfest sums per step and instance.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._device import ptr, require_cuda, stream_handle, to_device
from ._lib import FW_F32, FW_F64, FW_STEP_FUSED, WignerDesc, check


class WignerMoyalBatch:
    def __init__(self, *, batch, X_gridDIM, X_amplitude, P_gridDIM, P_amplitude, dt, V, K, diff_V=None,
                 diff_K=None, t=0.0, hbar=1.0, precision="float32", observables=True):
        self.batch = int(batch)
        self.X_gridDIM, self.P_gridDIM = int(X_gridDIM), int(P_gridDIM)
        self.X_amplitude, self.P_amplitude = float(X_amplitude), float(P_amplitude)
        self.dt, self.t, self.hbar = float(dt), float(t), float(hbar)
        self.precision = precision
        f64 = precision == "float64"
        self._rt = torch.float64 if f64 else torch.float32
        self._ct = torch.complex128 if f64 else torch.complex64
        self._code = FW_F64 if f64 else FW_F32
        Xn, Pn = self.X_gridDIM, self.P_gridDIM
        self.dX = 2.0 * self.X_amplitude / Xn
        self.dP = 2.0 * self.P_amplitude / Pn
        self.dXdP = self.dX * self.dP
        self.X = np.linspace(-self.X_amplitude, self.X_amplitude - self.dX, Xn)[np.newaxis, :]
        self.P = np.linspace(-self.P_amplitude, self.P_amplitude - self.dP, Pn)[:, np.newaxis]
        self.Lambda = np.fft.fftfreq(Xn, self.dX / (2 * np.pi))[: Xn // 2 + 1][np.newaxis, :]
        self.Theta = np.fft.fftfreq(Pn, self.dP / (2 * np.pi))[: Pn // 2 + 1][:, np.newaxis]
        self.device = require_cuda()
        self._lib = _lib.load()
        self._plan = _lib.c_vp()
        check(self._lib.fw_wigner_plan_create(Pn, Xn, self.batch, self._code, ctypes.byref(self._plan)),
              "fw_wigner_plan_create")
        Vs = V if isinstance(V, (list, tuple)) else [V]
        Ks = K if isinstance(K, (list, tuple)) else [K]
        if len(Vs) != len(Ks) or len(Vs) not in (1, self.batch):
            raise ValueError("V and K must be one callable each or lists of length batch")
        self.per_instance = len(Vs) > 1
        h = self.hbar
        Xm, Xp = self.X - 0.5 * h * self.Theta, self.X + 0.5 * h * self.Theta
        Pp, Pm = self.P + 0.5 * h * self.Lambda, self.P - 0.5 * h * self.Lambda
        tv, tk = [], []
        for v, k in zip(Vs, Ks):
            tv.append(np.broadcast_to(np.exp(-0.5j * dt / h * (v(Xm) - v(Xp))), Xm.shape))
            tk.append(np.broadcast_to(np.exp(-1j * dt / h * (k(Pp) - k(Pm))), Pp.shape))
        self._tabV = torch.view_as_real(to_device(np.stack(tv), self._ct, self.device)).contiguous()
        self._tabK = torch.view_as_real(to_device(np.stack(tk), self._ct, self.device)).contiguous()
        self._tab_bstride = (self._tabV[0].numel() // 2) if self.per_instance else 0
        if self.per_instance and self._tabK[0].numel() // 2 != self._tab_bstride:
            # one stride serves both tables only for square spectra layouts; keep them in separate calls otherwise
            if (Pn // 2 + 1) * Xn != Pn * (Xn // 2 + 1):
                raise ValueError("per-instance tables need P_gridDIM == X_gridDIM")
        self._M = 2
        self._wx = self._wp = None
        if observables and diff_V is not None and diff_K is not None:
            wx = np.stack([self.X[0], np.broadcast_to(diff_V(self.X), self.X.shape)[0],
                           np.broadcast_to(Vs[0](self.X), self.X.shape)[0]])
            wp = np.stack([self.P[:, 0], np.broadcast_to(diff_K(self.P), self.P.shape)[:, 0],
                           np.broadcast_to(Ks[0](self.P), self.P.shape)[:, 0]])
            self._wx = to_device(wx, torch.float64, self.device)
            self._wp = to_device(wp, torch.float64, self.device)
            self._M = 8
        self.W = torch.zeros((self.batch, Pn, Xn), dtype=self._rt, device=self.device)

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                self._lib.fw_wigner_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def set_wignerfunctions(self, W):
        """Copy B states (host array / tensor, B x P x X) and normalise each."""
        if isinstance(W, torch.Tensor):
            self.W.copy_(W, non_blocking=True)
        else:
            self.W.copy_(torch.as_tensor(np.asarray(W)).to(self._rt))
        s = self.W.sum(dim=(1, 2), dtype=torch.float64) * self.dXdP
        self.W.div_(s.to(self._rt)[:, None, None])
        return self

    def _desc(self, obs):
        d = WignerDesc()
        d.W = ptr(self.W)
        d.w_bstride = self.P_gridDIM * self.X_gridDIM
        d.step_kind = FW_STEP_FUSED
        d.tabV, d.tabK = ptr(self._tabV), ptr(self._tabK)
        d.tabV_step = d.tabK_step = 0
        d.tab_bstride = self._tab_bstride
        d.tab_real = 0
        if self._wx is not None:
            d.Mx = d.Mp = 3
            d.wx, d.wp = ptr(self._wx), ptr(self._wp)
        d.obs_out = ptr(obs)
        d.dxdp = self.dXdP
        d.in_scale = 1.0
        return d

    def propagate(self, steps=1, obs=None):
        """Advance all instances; returns the device tensor of observable sums
        (steps x batch x M: [sum W, sum W^2, <x>, <V'>, <V>, <p>, <K'>, <K>] sums)."""
        if obs is None:
            obs = torch.empty((steps, self.batch, self._M), dtype=torch.float64, device=self.device)
        d = self._desc(obs)
        check(self._lib.fw_wigner_propagate(self._plan, ctypes.byref(d), int(steps), stream_handle()),
              "fw_wigner_propagate")
        self.t += steps * self.dt
        return obs

    def propagate_host_batches(self, states, steps, out=None, obs_out=None):
        """Propagate a sequence of host-resident batches (each B x P x X; pinned
        CPU tensors copy asynchronously) by `steps` steps each, every batch from
        the current time.  Batch i is copied in, normalised as by
        set_wignerfunctions, propagated, and copied back to out[i] (host, same
        shape) with its observable sums (steps x B x M) in obs_out[i] when given.
        The copies in and out run on their own streams into two alternating
        device state buffers, so they overlap the propagation of the
        neighbouring batches.  out[i] may repeat tensors (the caller reuses
        host buffers); everything is complete when the current stream is.
        Afterwards self.W holds the last batch's final states.
        Returns (out, obs_out)."""
        n = len(states)
        if out is None:
            out = [torch.empty(self.W.shape, dtype=self._rt).pin_memory() for _ in range(n)]
        if getattr(self, "_W_alt", None) is None or self._W_alt.shape != self.W.shape:
            self._W_alt = torch.empty_like(self.W)
        bufs = [self.W, self._W_alt]
        obs_dev = [torch.empty((steps, self.batch, self._M), dtype=torch.float64, device=self.device)
                   for _ in range(2)]
        comp = torch.cuda.current_stream(self.device)
        h2d, d2h = torch.cuda.Stream(self.device), torch.cuda.Stream(self.device)
        h2d.wait_stream(comp)  # earlier work on the buffers comes first
        free = [None, None]    # per buffer: its last copy-out has finished
        t0 = self.t
        for i in range(n):
            k = i & 1
            buf = bufs[k]
            with torch.cuda.stream(h2d):
                if free[k] is not None:
                    h2d.wait_event(free[k])
                buf.copy_(states[i], non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(h2d)
            comp.wait_event(loaded)
            s = buf.sum(dim=(1, 2), dtype=torch.float64) * self.dXdP
            buf.div_(s.to(self._rt)[:, None, None])
            self.W = buf
            self.t = t0
            self.propagate(steps, obs=obs_dev[k])
            done = torch.cuda.Event()
            done.record(comp)
            with torch.cuda.stream(d2h):
                d2h.wait_event(done)
                out[i].copy_(buf, non_blocking=True)
                if obs_out is not None:
                    obs_out[i].copy_(obs_dev[k], non_blocking=True)
                freed = torch.cuda.Event()
                freed.record(d2h)
            free[k] = freed
        for ev in free:  # the last copies-out complete before the caller's stream moves on
            if ev is not None:
                comp.wait_event(ev)
        self.t = t0 + steps * self.dt
        return out, obs_out

    def propagate_timed(self, steps=1):
        """propagate() with per-launch CUDA-event times: returns (obs, ms[], kind[])."""
        obs = torch.empty((steps, self.batch, self._M), dtype=torch.float64, device=self.device)
        d = self._desc(obs)
        n = 3 * steps + 4
        ms = (ctypes.c_float * n)()
        kind = (ctypes.c_int * n)()
        check(self._lib.fw_wigner_propagate_timed(self._plan, ctypes.byref(d), int(steps), stream_handle(), ms,
                                                  kind, n), "fw_wigner_propagate_timed")
        self.t += steps * self.dt
        nl = 2 * steps + 2
        return obs, np.array(ms[:nl]), np.array(kind[:nl])


# =============================================================================
# Uneven batches: one persistent launch over instances of different grid sizes
# =============================================================================
def _autotune_path():
    import os
    from pathlib import Path

    p = os.environ.get("FASTWIGNER_AUTOTUNE")
    return Path(p) if p else Path.home() / ".cache" / "fastwigner_b200" / "autotune.json"


class WignerMoyalUnevenBatch:
    """Independent FP32 Moyal instances with their own grids (P, X in
    {128, 256, 512, 1024}), amplitudes and Hamiltonians.  Conventions are
    WignerMoyalFTTW1D's (static Hamiltonians; exponents as in
    wigner_moyal_fftw_1d.py:164-213).  Two execution modes, both optionally
    replayed as a CUDA graph:

    * variants 0 .. GROUPED-1: one persistent cooperative launch per
      ``propagate`` call over every instance, in one of the launch shapes;
    * GROUPED: instances of one (P, X, dX dP) share one state buffer, one
      table buffer and one plan of the single-shape path, and the groups run
      one after another (the persistent pass kernels where a group is large
      enough, the regular ones otherwise).

    ``specs``: one dict per instance with X_gridDIM, P_gridDIM, X_amplitude,
    P_amplitude, V (callable of x), K (callable of p).  ``variant`` None picks
    the mode with the autotuner (timings cached in a JSON file keyed by GPU
    and size mix, the analogue of FFTW wisdom).  ``W[i]`` is instance i's
    state (a view into its group's buffer, shared by both modes)."""

    def __init__(self, specs, *, dt, t=0.0, hbar=1.0, variant=None, autotune_steps=10):
        self.dt, self.t, self.hbar = float(dt), float(t), float(hbar)
        self.device = require_cuda()
        self._lib = _lib.load()
        self.specs = [dict(s) for s in specs]
        n = len(self.specs)
        P = (ctypes.c_int * n)(*[int(s["P_gridDIM"]) for s in self.specs])
        X = (ctypes.c_int * n)(*[int(s["X_gridDIM"]) for s in self.specs])
        self._h = _lib.c_vp()
        check(self._lib.fw_batch_create(n, P, X, 0, ctypes.byref(self._h)), "fw_batch_create")
        self.GROUPED = self._lib.fw_batch_num_variants()  # the variant index of the grouped mode
        self._groups = self._make_groups()
        self.W, self._tabs, self.dXdP = [None] * n, [None] * n, [None] * n
        for i, s in enumerate(self.specs):
            Pn, Xn = int(s["P_gridDIM"]), int(s["X_gridDIM"])
            dX, dP = 2.0 * s["X_amplitude"] / Xn, 2.0 * s["P_amplitude"] / Pn
            x = np.linspace(-s["X_amplitude"], s["X_amplitude"] - dX, Xn)[None, :]
            p = np.linspace(-s["P_amplitude"], s["P_amplitude"] - dP, Pn)[:, None]
            th = np.fft.fftfreq(Pn, dP / (2 * np.pi))[: Pn // 2 + 1][:, None]
            la = np.fft.fftfreq(Xn, dX / (2 * np.pi))[: Xn // 2 + 1][None, :]
            h = self.hbar
            ev = np.broadcast_to(np.exp(-0.5j * self.dt / h * (s["V"](x - 0.5 * h * th) - s["V"](x + 0.5 * h * th))),
                                 (Pn // 2 + 1, Xn))
            ek = np.broadcast_to(np.exp(-1j * self.dt / h * (s["K"](p + 0.5 * h * la) - s["K"](p - 0.5 * h * la))),
                                 (Pn, Xn // 2 + 1))
            # the instance's state and tables are slices of its shape group's
            # buffers, which the grouped mode propagates as one plan
            g, k = self._slot[i]
            W = g["W"][k]
            tv, tk = g["tab"][2 * k], g["tab"][2 * k + 1]
            tv[: ev.size].copy_(to_device(np.ascontiguousarray(ev).ravel(), torch.complex64, self.device))
            tk[: ek.size].copy_(to_device(np.ascontiguousarray(ek).ravel(), torch.complex64, self.device))
            self.W[i] = W
            self._tabs[i] = (tv, tk)
            self.dXdP[i] = dX * dP
            s.update(X=x, P=p, dX=dX, dP=dP)
            check(self._lib.fw_batch_set_instance(self._h, i, ptr(W), ptr(tv), ptr(tk), dX * dP),
                  "fw_batch_set_instance")
        self._graph = None
        self._graph_key = None
        self.variant = 0
        if variant is None:
            variant = self.autotune(autotune_steps)
        self.set_variant(variant)

    def _make_groups(self):
        """Instances of equal (P, X, dX dP), in order of first appearance: one
        state buffer (n x P x X), one table buffer (2n slots of S complex
        entries, V table then K table per instance, S the larger table rounded
        to an even count so every slot starts on 16 bytes) and one plan each."""
        from ._lib import FW_F32

        keys, members = [], {}
        for i, s in enumerate(self.specs):
            Pn, Xn = int(s["P_gridDIM"]), int(s["X_gridDIM"])
            dxdp = (2.0 * s["X_amplitude"] / Xn) * (2.0 * s["P_amplitude"] / Pn)
            key = (Pn, Xn, dxdp)
            if key not in members:
                keys.append(key)
                members[key] = []
            members[key].append(i)
        groups, self._slot = [], {}
        for key in keys:
            Pn, Xn, dxdp = key
            idx = members[key]
            S = max((Pn // 2 + 1) * Xn, Pn * (Xn // 2 + 1))
            S += S % 2
            g = {"P": Pn, "X": Xn, "dxdp": dxdp, "idx": idx, "S": S,
                 "idx_t": torch.tensor(idx, dtype=torch.long, device=self.device),
                 "W": torch.zeros((len(idx), Pn, Xn), dtype=torch.float32, device=self.device),
                 "tab": torch.zeros((2 * len(idx), S), dtype=torch.complex64, device=self.device),
                 "plan": _lib.c_vp()}
            check(self._lib.fw_wigner_plan_create(Pn, Xn, len(idx), FW_F32, ctypes.byref(g["plan"])),
                  "fw_wigner_plan_create")
            for k, i in enumerate(idx):
                self._slot[i] = (g, k)
            groups.append(g)
        return groups

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.fw_batch_destroy(h)
            except Exception:
                pass
            self._h = None
        self._graph = None
        for g in getattr(self, "_groups", []):
            if g["plan"].value:
                try:
                    self._lib.fw_wigner_plan_destroy(g["plan"])
                except Exception:
                    pass
                g["plan"].value = None

    def set_variant(self, v):
        """0, 1: launch shapes of the persistent cooperative kernel; GROUPED:
        one plan per shape group (the regular and persistent pass kernels of
        the single-shape path, all groups replayed as one CUDA graph)."""
        if not 0 <= int(v) <= self.GROUPED:
            raise ValueError(f"variant must be in [0, {self.GROUPED}]")
        if int(v) != self.GROUPED:
            check(self._lib.fw_batch_set_variant(self._h, int(v)), "fw_batch_set_variant")
            self._graph = self._graph_key = self._graph_obs = None
        self.variant = int(v)

    def set_wignerfunctions(self, states):
        """One state per instance (array / tensor of that instance's shape); each is normalised."""
        for W, s, d in zip(self.W, states, self.dXdP):
            W.copy_(to_device(s, torch.float32, self.device) if not isinstance(s, torch.Tensor) else s)
            W.div_(float(W.sum(dtype=torch.float64)) * d)
        return self

    def propagate(self, steps=1, use_graph=True, obs=None):
        """Advance every instance; returns the device tensor of per-step sums
        (steps x ninst x 2: sum W, sum W^2)."""
        if obs is None:
            obs = torch.empty((steps, len(self.specs), 2), dtype=torch.float64, device=self.device)
        if self.variant == self.GROUPED:
            self._propagate_grouped(int(steps), use_graph, obs)
        else:
            check(self._lib.fw_batch_propagate(self._h, int(steps), ptr(obs), 1 if use_graph else 0,
                                               stream_handle()), "fw_batch_propagate")
        self.t += steps * self.dt
        return obs

    def _launch_groups(self, steps, obs, obs_g):
        from ._lib import FW_STEP_FUSED

        # the groups one after another on the current stream: replayed from a
        # graph, the small groups' launches are short enough that side streams
        # gained nothing over this order (0.669 vs 0.668 ms per step for the
        # 256-instance mix of 16 shapes) and a multi-stream graph lost 17 %
        for g, og in zip(self._groups, obs_g):
            d = WignerDesc()
            d.W = ptr(g["W"])
            d.w_bstride = g["P"] * g["X"]
            d.step_kind = FW_STEP_FUSED
            d.tabV, d.tabK = ptr(g["tab"][0]), ptr(g["tab"][1])
            d.tab_bstride = 2 * g["S"]
            d.obs_out = ptr(og)
            d.dxdp = g["dxdp"]
            d.in_scale = 1.0
            check(self._lib.fw_wigner_propagate(g["plan"], ctypes.byref(d), steps, stream_handle()),
                  "fw_wigner_propagate")
        for g, og in zip(self._groups, obs_g):
            obs.index_copy_(1, g["idx_t"], og)

    def _propagate_grouped(self, steps, use_graph, obs):
        if not use_graph:
            obs_g = [torch.empty((steps, len(g["idx"]), 2), dtype=torch.float64, device=self.device)
                     for g in self._groups]
            self._launch_groups(steps, obs, obs_g)
            return
        key = (steps, obs.data_ptr())
        if self._graph_key != key:
            self._graph = None
            obs_g = [torch.empty((steps, len(g["idx"]), 2), dtype=torch.float64, device=self.device)
                     for g in self._groups]
            self._launch_groups(steps, obs, obs_g)  # first call direct: one-time set-up outside the capture
            torch.cuda.synchronize(self.device)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                self._launch_groups(steps, obs, obs_g)
            self._graph, self._graph_key, self._graph_obs = graph, key, obs_g
            # the direct call above already advanced the states by `steps`
            return
        self._graph.replay()

    def status(self):
        """The persistent kernel's device status word (FW_BATCH_TIMEOUT after an
        expired grid barrier), or else the first non-zero status of the
        grouped mode's plans."""
        st = ctypes.c_int()
        check(self._lib.fw_batch_status(self._h, ctypes.byref(st)), "fw_batch_status")
        for g in self._groups:
            if st.value:
                break
            check(self._lib.fw_wigner_plan_status(g["plan"], ctypes.byref(st), 0), "fw_wigner_plan_status")
        return st.value

    def set_status(self, value=0):
        """Write the device status word: 0 clears a recorded FW_BATCH_TIMEOUT;
        a non-zero value makes the next launch return at its first grid barrier."""
        check(self._lib.fw_batch_set_status(self._h, int(value)), "fw_batch_set_status")

    def set_spin_limit(self, polls):
        """Polls a CTA waits at a grid barrier before the launch gives up with
        FW_BATCH_TIMEOUT (default 2**25, a few seconds)."""
        check(self._lib.fw_batch_set_spin_limit(self._h, int(polls)), "fw_batch_set_spin_limit")

    def purity(self, obs):
        """2 pi hbar sum(W^2) dXdP of the normalised states, from propagate()'s sums."""
        o = obs.cpu().numpy() if isinstance(obs, torch.Tensor) else obs
        d = np.array(self.dXdP)
        return 2 * np.pi * self.hbar * o[..., 1] / (o[..., 0] ** 2 * d)

    # -- autotuner ----------------------------------------------------------------
    def _key(self):
        import collections

        hist = collections.Counter((int(s["P_gridDIM"]), int(s["X_gridDIM"])) for s in self.specs)
        mix = ",".join(f"{p}x{x}:{c}" for (p, x), c in sorted(hist.items()))
        return f"{torch.cuda.get_device_name(self.device)}|{mix}"

    def autotune(self, steps=10, cache=True):
        """Time every launch-shape variant on this batch (states are saved and
        restored) and return the fastest; results are cached per GPU and size mix."""
        import json

        path = _autotune_path()
        key = self._key()
        if cache and path.exists():
            try:
                table = json.loads(path.read_text())
                if key in table:
                    return int(table[key]["variant"])
            except (ValueError, KeyError, OSError):
                pass
        saved = [g["W"].clone() for g in self._groups]
        t_saved = self.t
        times = {}
        obs = torch.empty((steps, len(self.specs), 2), dtype=torch.float64, device=self.device)
        for v in range(self.GROUPED + 1):
            # each mode as propagate(use_graph=True) runs it: the first call
            # captures the graph, the second replays it
            self.set_variant(v)
            self.propagate(steps, use_graph=True, obs=obs)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.propagate(steps, use_graph=True, obs=obs)
            e1.record()
            torch.cuda.synchronize()
            times[v] = e0.elapsed_time(e1) / steps
        self._graph = self._graph_key = self._graph_obs = None
        for g, s in zip(self._groups, saved):
            g["W"].copy_(s)
        self.t = t_saved
        best = min(times, key=times.get)
        if cache:
            try:
                path.parent.mkdir(parents=True, exist_ok=True)
                table = json.loads(path.read_text()) if path.exists() else {}
                table[key] = {"variant": best, "ms_per_step": times}
                path.write_text(json.dumps(table, indent=1))
            except OSError:
                pass
        self.autotune_ms = times
        return best
