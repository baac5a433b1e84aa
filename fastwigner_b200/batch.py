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
