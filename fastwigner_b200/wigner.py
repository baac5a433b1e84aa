"""Drop-in Wigner-function split-operator propagators running on B200.

Classes (same constructor keywords, attributes and methods as the reference):

* ``WignerMoyalFTTW1D``  -- wigner_moyal_fftw_1d.py:6   (numpy callables)
* ``WignerBlochFFTW1D``  -- wigner_bloch_fftw_1d.py:6
* ``WignerRandomCollisionModelFFTW1D`` -- wigner_random_collision_model_fftw_1d.py:6
* ``WignerMoyalCUDA1D``  -- wigner_moyal_cuda_1d.py:10  (C-expression strings)
* ``WignerBlochCUDA1D``  -- wigner_bloch_cuda_1d.py:8

The state lives on the GPU as a torch tensor; every step runs as two fused
passes of libfastwigner (column pass: FFT_p -> exp(V) -> iFFT_p [-> observables
-> FFT_p -> exp(V) -> iFFT_p], row pass: FFT_x -> exp(K) -> iFFT_x).  The
phase tables are evaluated in FP64 (host numpy for callables, NVRTC-compiled
device code for C strings) exactly where the reference evaluates them and
stored in the working precision (``precision="float64"`` default, or
``"float32"`` for complex64 spectra with FP64-built phases).

Extensions beyond the reference: ``hbar`` (default 1) and ``precision``.
"""
from __future__ import annotations

from types import FunctionType, MethodType

import numpy as np
import torch

from . import _lib
from ._device import DeviceArray, ptr, require_cuda, stream_handle, to_device
from ._lib import FW_F32, FW_F64, FW_STEP_FUSED, FW_STEP_SPLIT, FastWignerError, WignerDesc, check

# at most this many time-dependent phase tables are materialised per launch
_TD_CHUNK_BYTES = 256 << 20


def _bind_kwargs(obj, kwargs):
    """Bind keyword arguments as the reference does: functions become methods
    (wigner_moyal_fftw_1d.py:41-47), everything else an attribute."""
    for name, value in kwargs.items():
        if isinstance(value, FunctionType):
            setattr(obj, name, MethodType(value, obj))
        else:
            setattr(obj, name, value)


def _require(obj, name, msg):
    try:
        getattr(obj, name)
    except AttributeError:
        raise AttributeError(msg) from None


class _WignerBase:
    """Shared machinery: grids, tables, plan, step sequencing, observables."""

    _conv = "fftw"  # grid / time conventions: "fftw" or "cuda"

    # -- construction -------------------------------------------------------
    def __init__(self, **kwargs):
        _bind_kwargs(self, kwargs)
        self._kwargs = dict(kwargs)
        _require(self, "X_gridDIM", "Coordinate grid size (X_gridDIM) was not specified")
        assert self.X_gridDIM % 2 == 0, "Coordinate grid size (X_gridDIM) must be even"
        _require(self, "P_gridDIM", "Momentum grid size (P_gridDIM) was not specified")
        assert self.P_gridDIM % 2 == 0, "Momentum grid size (P_gridDIM) must be even"
        _require(self, "X_amplitude", "Coordinate grid range (X_amplitude) was not specified")
        _require(self, "P_amplitude", "Momentum grid range (P_amplitude) was not specified")
        _require(self, "V", "Potential energy (V) was not specified")
        _require(self, "K", "Momentum dependence (K) was not specified")
        _require(self, "dt", "Time-step (dt) was not specified")
        try:
            self.t
        except AttributeError:
            print("Warning: Initial time (t) was not specified, thus it is set to zero.")
            self.t = 0.0
        self.t = float(self.t)
        self.hbar = float(getattr(self, "hbar", 1.0))
        prec = str(getattr(self, "precision", "float64"))
        if prec not in ("float64", "float32"):
            raise ValueError("precision must be 'float64' or 'float32'")
        self.precision = prec
        self._f64 = prec == "float64"
        self._rt = torch.float64 if self._f64 else torch.float32
        self._ct = torch.complex128 if self._f64 else torch.complex64
        self._code = FW_F64 if self._f64 else FW_F32
        self._make_grids()
        self.device = require_cuda()
        self._lib = _lib.load()
        self._plan = _lib.c_vp()
        check(self._lib.fw_wigner_plan_create(self.P_gridDIM, self.X_gridDIM, 1, self._code,
                                              _lib.ctypes.byref(self._plan)), "fw_wigner_plan_create")
        self._W = torch.zeros((self.P_gridDIM, self.X_gridDIM), dtype=self._rt, device=self.device)
        self._host_cache = None
        self._step_kind = FW_STEP_FUSED
        self._s0 = None
        self._blend_c = 1.0
        self._bxp = None

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                self._lib.fw_wigner_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def _make_grids(self):
        """wigner_moyal_fftw_1d.py:101-127 (FFTW) / wigner_moyal_cuda_1d.py:113-143 (CUDA)."""
        X, P = self.X_gridDIM, self.P_gridDIM
        self.dX = 2.0 * self.X_amplitude / X
        self.dP = 2.0 * self.P_amplitude / P
        self.dXdP = self.dX * self.dP
        lam = np.fft.fftfreq(X, self.dX / (2 * np.pi))
        th = np.fft.fftfreq(P, self.dP / (2 * np.pi))
        self.dLambda = lam[1] - lam[0]
        self.dTheta = th[1] - th[0]
        self.X = np.linspace(-self.X_amplitude, self.X_amplitude - self.dX, X)[np.newaxis, :]
        self.P = np.linspace(-self.P_amplitude, self.P_amplitude - self.dP, P)[:, np.newaxis]
        self.Lambda = lam[: X // 2 + 1][np.newaxis, :]
        self.Theta = th[: P // 2 + 1][:, np.newaxis]
        if self._conv == "cuda":
            # the CUDA kernels index the grids as dX*(j - X/2), dLambda*j (positive Nyquist)
            self._Xk = (self.dX * (np.arange(X) - 0.5 * X))[np.newaxis, :]
            self._Pk = (self.dP * (np.arange(P) - 0.5 * P))[:, np.newaxis]
            self._Lk = (self.dLambda * np.arange(X // 2 + 1))[np.newaxis, :]
            self._Tk = (self.dTheta * np.arange(P // 2 + 1))[:, np.newaxis]
        else:
            self._Xk, self._Pk, self._Lk, self._Tk = self.X, self.P, self.Lambda, self.Theta
        h = self.hbar
        self.X_minus = self._Xk - 0.5 * h * self._Tk
        self.X_plus = self._Xk + 0.5 * h * self._Tk
        self.P_minus = self._Pk - 0.5 * h * self._Lk
        self.P_plus = self._Pk + 0.5 * h * self._Lk

    # -- hooks the subclasses provide ---------------------------------------
    def _v_at(self, x, t):  # V on an array of coordinates at time t (FP64 numpy)
        raise NotImplementedError

    def _k_at(self, p, t):
        raise NotImplementedError

    def _v_time_dependent(self) -> bool:
        raise NotImplementedError

    def _k_time_dependent(self) -> bool:
        raise NotImplementedError

    def _phase_time(self, t):
        """Time at which the exponents of the step ending at t are evaluated."""
        return t + 0.5 * self.dt if self._conv == "cuda" else t

    # -- tables ---------------------------------------------------------------
    def _exp_v_host(self, t):
        """exp(-i dt/(2 hbar) [V(x - hbar theta/2) - V(x + hbar theta/2)]) * boundary, (P/2+1) x X."""
        ph = -0.5 * self.dt / self.hbar * (self._v_at(self.X_minus, t) - self._v_at(self.X_plus, t))
        e = np.exp(1j * ph)
        return e * self._b_x_theta()

    def _exp_k_host(self, t):
        """exp(-i dt/hbar [K(p + hbar lambda/2) - K(p - hbar lambda/2)]) * boundary, P x (X/2+1)."""
        ph = -self.dt / self.hbar * (self._k_at(self.P_plus, t) - self._k_at(self.P_minus, t))
        return np.exp(1j * ph) * self._b_lambda_p()

    def _b_x_theta(self):
        return 1.0

    def _b_lambda_p(self):
        return 1.0

    def _tables_static(self) -> bool:
        return not (self._v_time_dependent() or self._k_time_dependent())

    def _upload_table(self, a, shape, real=None):
        a = np.broadcast_to(a, shape)
        if real is None:
            real = bool(getattr(self, "_tab_real", False))
        if real:
            return to_device(np.real(a), self._rt, self.device)
        return torch.view_as_real(to_device(a, self._ct, self.device)).contiguous()

    def _static_tables(self):
        if getattr(self, "_tabV_dev", None) is None:
            t = self._phase_time(self.t)
            self._tabV_dev = self._upload_table(self._exp_v_host(t), self.X_minus.shape)
            self._tabK_dev = self._upload_table(self._exp_k_host(t), self.P_plus.shape)
        return self._tabV_dev, self._tabK_dev

    # -- observables ------------------------------------------------------------
    def _obs_weights(self, times):
        """x- and p-weights of the Ehrenfest observables per step: Mx x X, Mp x P."""
        if not self.isEhrenfest:
            return None, None
        raise NotImplementedError

    def _ehrenfest_from_obs(self, obs):
        S = obs[:, 0]
        xw = obs[:, 2:5]
        pw = obs[:, 5:8]
        self.X_average.extend((xw[:, 0] / S).tolist())
        self.P_average_RHS.extend((-xw[:, 1] / S).tolist())
        self.P_average.extend((pw[:, 0] / S).tolist())
        self.X_average_RHS.extend((pw[:, 1] / S).tolist())
        self.hamiltonian_average.extend(((pw[:, 2] + xw[:, 2]) / S).tolist())

    # -- state ----------------------------------------------------------------
    def _normalise_(self):
        s = float(self._W.sum(dtype=torch.float64)) * self.dXdP
        self._W.div_(s)
        self._host_cache = None

    def _set_state_array(self, a):
        if isinstance(a, DeviceArray):
            a = a.tensor
        shape = tuple(a.shape)
        assert shape == (self.P_gridDIM, self.X_gridDIM), "The grid sizes does not match with the Wigner function"
        if isinstance(a, torch.Tensor):
            assert not a.is_complex() and a.is_floating_point(), "Supplied Wigner function must be real"
            self._W.copy_(a.to(self._rt))
        else:
            a = np.asarray(a)
            assert np.issubdtype(a.dtype, np.floating), "Supplied Wigner function must be real"
            self._W.copy_(to_device(a, self._rt, self.device))

    @property
    def wigner_device(self) -> torch.Tensor:
        """The live device tensor holding W (P x X)."""
        return self._W

    # -- propagation ------------------------------------------------------------
    def _propagate_chunk(self, nsteps, t0, tables=None, weights=None, host=True):
        """Run nsteps steps starting after time t0; return the observable sums
        (nsteps x M; a numpy copy, or the device tensor when host is False).

        tables: optional (tabV, vstep, tabK, kstep, tab_real) overriding the
        Hamiltonian's phase tables; weights: optional (wx, wp) overriding the
        Ehrenfest weights (use (None, None) for none)."""
        times = t0 + self.dt * np.arange(1, nsteps + 1)
        if tables is not None:
            tabV, vstep, tabK, kstep, tab_real = tables
        else:
            tab_real = bool(getattr(self, "_tab_real", False))
            if self._tables_static():
                tabV, tabK = self._static_tables()
                vstep = kstep = 0
            else:
                tabV, vstep = self._td_tables(times, "V")
                tabK, kstep = self._td_tables(times, "K")
        wx, wp = self._obs_weights(times) if weights is None else weights
        Mx = 0 if wx is None else wx.shape[-2]
        Mp = 0 if wp is None else wp.shape[-2]
        M = 2 + Mx + Mp
        obs = torch.empty((nsteps, M), dtype=torch.float64, device=self.device)
        d = WignerDesc()
        d.W = ptr(self._W)
        d.w_bstride = self._W.numel()
        d.step_kind = self._step_kind
        d.tabV, d.tabV_step = ptr(tabV), vstep
        d.tabK, d.tabK_step = ptr(tabK), kstep
        d.tab_bstride = 0
        d.tab_real = 1 if tab_real else 0
        gV, gK = getattr(self, "_gV", None), getattr(self, "_gK", None)
        if gV is not None:  # separable per-step factors over theta / lambda (complex, steps x len x 2)
            d.gV, d.gV_step = ptr(gV), gV.shape[-2]
        if gK is not None:
            d.gK, d.gK_step = ptr(gK), gK.shape[-2]
        d.bxp = ptr(self._bxp)
        d.s0 = ptr(self._s0)
        d.blend_c = self._blend_c
        d.Mx, d.Mp = Mx, Mp
        if wx is not None:
            d.wx = ptr(wx)
            d.wx_step = wx.shape[-1] * Mx if wx.dim() == 3 else 0
        if wp is not None:
            d.wp = ptr(wp)
            d.wp_step = wp.shape[-1] * Mp if wp.dim() == 3 else 0
        d.obs_out = ptr(obs)
        d.dxdp = self.dXdP
        d.in_scale = 1.0
        check(self._lib.fw_wigner_propagate(self._plan, _lib.ctypes.byref(d), nsteps, stream_handle()),
              "fw_wigner_propagate")
        self._host_cache = None
        return obs.cpu().numpy() if host else obs

    def _chunk_context(self):
        """Host-side state of the last chunk that _ehrenfest_from_obs needs, for
        chunks whose observables are processed later (propagate with frames)."""
        return None

    def _set_chunk_context(self, ctx):
        pass

    def _td_tables(self, times, which):
        td = self._v_time_dependent() if which == "V" else self._k_time_dependent()
        if not td:
            tabV, tabK = self._static_tables_partial(which)
            return (tabV if which == "V" else tabK), 0
        shape = self.X_minus.shape if which == "V" else self.P_plus.shape
        build = self._exp_v_host if which == "V" else self._exp_k_host
        tabs = np.stack([np.broadcast_to(build(self._phase_time(t)), shape) for t in times])
        dev = self._upload_table(tabs, tabs.shape)
        per = int(np.prod(shape))
        return dev, per

    def _static_tables_partial(self, which):
        key = "_tab%s_static" % which
        if getattr(self, key, None) is None:
            t = self._phase_time(self.t)
            if which == "V":
                setattr(self, key, self._upload_table(self._exp_v_host(t), self.X_minus.shape))
            else:
                setattr(self, key, self._upload_table(self._exp_k_host(t), self.P_plus.shape))
        return (getattr(self, key), None) if which == "V" else (None, getattr(self, key))

    def _chunk_steps(self):
        if self._tables_static():
            return 1 << 30
        per = (self.X_minus.size + self.P_plus.size) * (8 if not self._f64 else 16)
        return max(1, _TD_CHUNK_BYTES // per)

    def propagate(self, steps=1, frames=None, frame_every=0):
        """Advance by `steps` time steps, renormalising and recording the
        Ehrenfest observables after each (wigner_moyal_fftw_1d.py:418-440).

        The steps run in chunks (per-step tables or factor vectors are built on
        the host one chunk at a time) without waiting for the device between
        chunks, so the host prepares a chunk while the previous one runs; the
        Ehrenfest lists are filled from every chunk's sums before returning.

        Extension: with a FrameRecorder `frames` and frame_every = k > 0 the
        state is recorded (``frames.record(t=..., wigner=<device state>)``)
        after every k steps."""
        steps = int(steps)
        every = int(frame_every) if frames is not None else 0
        done = 0
        pending = []
        while done < steps:
            n = min(steps - done, self._chunk_steps())
            if every > 0:
                n = min(n, every - done % every)
            pending.append((self._propagate_chunk(n, self.t, host=False), self._chunk_context()))
            self.t += n * self.dt
            done += n
            if every > 0 and done % every == 0:
                frames.record(t=self.t, wigner=self.wigner_device)
        for obs, ctx in pending:
            obs = obs.cpu().numpy()
            self._set_chunk_context(ctx)
            self._last_obs = obs
            if self.isEhrenfest:
                self._ehrenfest_from_obs(obs)
        return self._returned_state()

    def single_step_propagation(self):
        """One step without the final renormalisation (wigner_moyal_fftw_1d.py:397-416).
        Time is not advanced, as in the reference."""
        obs = self._propagate_chunk(1, self.t - self.dt)
        self._W.mul_(float(obs[0, 0]) * self.dXdP * self._unnormalised_factor())
        self._host_cache = None
        return self._returned_state()

    def _unnormalised_factor(self):
        return 1.0

    def get_purity(self):
        """2 pi hbar sum(W^2) dX dP (wigner_moyal_cuda_1d.py:398-403), the sum
        of squares reduced in FP64 on the device by fw_wigner_weighted_sum."""
        out = torch.empty(2, dtype=torch.float64, device=self.device)
        check(self._lib.fw_wigner_weighted_sum(self._plan, ptr(self._W), self._W.numel(), None, ptr(out),
                                               stream_handle()), "fw_wigner_weighted_sum")
        return 2.0 * np.pi * self.hbar * float(out[1]) * self.dXdP

    def _grid_average(self, F):
        """sum(W * F) dXdP with F a P x X FP64 grid, reduced on the device."""
        Fd = to_device(np.broadcast_to(F, self._W.shape), torch.float64, self.device)
        out = torch.empty(2, dtype=torch.float64, device=self.device)
        check(self._lib.fw_wigner_weighted_sum(self._plan, ptr(self._W), self._W.numel(), ptr(Fd), ptr(out),
                                               stream_handle()), "fw_wigner_weighted_sum")
        return float(out[0]) * self.dXdP

    def get_sigma_x_sigma_p(self):
        """sqrt(var x * var p) (wigner_moyal_cuda_1d.py:405-415)."""
        X, P = self._Xk, self._Pk
        return np.sqrt((self._grid_average(X * X + 0 * P) - self._grid_average(X + 0 * P) ** 2)
                       * (self._grid_average(P * P + 0 * X) - self._grid_average(P + 0 * X) ** 2))


# =============================================================================
# FFTW-family drop-ins (numpy callables)
# =============================================================================
class WignerMoyalFTTW1D(_WignerBase):
    """Second-order split-operator propagator for the Moyal equation
    (drop-in for wigner_moyal_fftw_1d.py:6).  V(self, x[, t]) and K(self, p[, t])
    are numpy callables; time dependence is detected as in the reference
    (one-argument call raising TypeError, :164-213)."""

    _conv = "fftw"

    def __init__(self, **kwargs):
        super().__init__(**kwargs)
        self._v_td = self._detect_td(self.V, self.X_minus)
        self._k_td = self._detect_td(self.K, self.P_plus)
        # absorbing boundary (wigner_moyal_fftw_1d.py:135-156)
        self._abs = self._abs_boundary(self.dt)
        self._setup_ehrenfest()

    @staticmethod
    def _detect_td(f, arg):
        try:
            f(arg)
            return False
        except TypeError:
            return True

    def _abs_boundary(self, dt):
        try:
            alpha = self.alpha
        except AttributeError:
            return 1.0
        xmin = min(self.X_minus.min(), self.X_plus.min())
        xmax = max(self.X_minus.max(), self.X_plus.max())
        b = np.sin(np.pi * (self.X_plus - xmin) / (xmax - xmin))
        b = b * np.sin(np.pi * (self.X_minus - xmin) / (xmax - xmin))
        return np.abs(b) ** abs(alpha * dt)

    def _b_x_theta(self):
        return self._abs

    def _v_time_dependent(self):
        return self._v_td

    def _k_time_dependent(self):
        return self._k_td

    def _v_at(self, x, t):
        return np.asarray(self.V(x, t) if self._v_td else self.V(x), dtype=np.float64)

    def _k_at(self, p, t):
        return np.asarray(self.K(p, t) if self._k_td else self.K(p), dtype=np.float64)

    def get_exp_v(self, t):
        """The potential exponent at time t, as a numpy array (reference API)."""
        return np.broadcast_to(self._exp_v_host(t), self.X_minus.shape)

    def get_exp_k(self, t):
        return np.broadcast_to(self._exp_k_host(t), self.P_plus.shape)

    def _setup_ehrenfest(self):
        """wigner_moyal_fftw_1d.py:221-273."""
        try:
            self.diff_V
            self.diff_K
        except AttributeError:
            self.isEhrenfest = False
            return
        self._dv_td = self._detect_td(self.diff_V, self.X)
        self._dk_td = self._detect_td(self.diff_K, self.P)
        self.X_average, self.P_average = [], []
        self.X_average_RHS, self.P_average_RHS = [], []
        self.hamiltonian_average = []
        self.isEhrenfest = True
        self._wx_static = self._wp_static = None

    def _weights_at(self, t):
        X, P = self.X.reshape(-1), self.P.reshape(-1)
        dv = self.diff_V(self.X, t) if self._dv_td else self.diff_V(self.X)
        dk = self.diff_K(self.P, t) if self._dk_td else self.diff_K(self.P)
        wx = np.stack([X, np.broadcast_to(dv, self.X.shape).reshape(-1),
                       np.broadcast_to(self._v_at(self.X, t), self.X.shape).reshape(-1)])
        wp = np.stack([P, np.broadcast_to(dk, self.P.shape).reshape(-1),
                       np.broadcast_to(self._k_at(self.P, t), self.P.shape).reshape(-1)])
        return wx, wp

    def _obs_weights(self, times):
        if not self.isEhrenfest:
            return None, None
        td = self._v_td or self._k_td or self._dv_td or self._dk_td
        if not td:
            if self._wx_static is None:
                wx, wp = self._weights_at(self.t)
                self._wx_static = to_device(wx, torch.float64, self.device)
                self._wp_static = to_device(wp, torch.float64, self.device)
            return self._wx_static, self._wp_static
        pairs = [self._weights_at(t) for t in times]
        wx = to_device(np.stack([a for a, _ in pairs]), torch.float64, self.device)
        wp = to_device(np.stack([b for _, b in pairs]), torch.float64, self.device)
        return wx, wp

    def get_Ehrenfest(self, t):
        """Record the Ehrenfest observables of the current state at time t
        (wigner_moyal_fftw_1d.py:442-481); returns the (coordinate, momentum) densities."""
        if not self.isEhrenfest:
            return None
        W = self._W.double()
        dc = W.sum(dim=0).cpu().numpy()
        dc /= dc.sum()
        dm = W.sum(dim=1).cpu().numpy()
        dm /= dm.sum()
        wx, wp = self._weights_at(t)
        self.X_average.append(np.dot(dc, wx[0]))
        self.P_average_RHS.append(-np.dot(dc, wx[1]))
        self.P_average.append(np.dot(dm, wp[0]))
        self.X_average_RHS.append(np.dot(dm, wp[1]))
        self.hamiltonian_average.append(np.dot(dm, wp[2]) + np.dot(dc, wx[2]))
        return dc, dm

    def set_wignerfunction(self, new_wigner_func):
        """Set the initial Wigner function from an array (numpy or torch, P x X)
        or a function F(self, X, P); then normalise (wigner_moyal_fftw_1d.py:368-395)."""
        if isinstance(new_wigner_func, (np.ndarray, torch.Tensor, DeviceArray)):
            self._set_state_array(new_wigner_func)
        elif isinstance(new_wigner_func, (FunctionType, MethodType)) or callable(new_wigner_func):
            f = new_wigner_func
            val = f(self, self.X, self.P) if isinstance(f, FunctionType) else f(self.X, self.P)
            self._set_state_array(np.broadcast_to(np.asarray(val, dtype=np.float64),
                                                  (self.P_gridDIM, self.X_gridDIM)))
        else:
            raise NotImplementedError("new_wigner_func must be either function or numpy.array")
        self._normalise_()
        return self

    @property
    def wignerfunction(self) -> np.ndarray:
        """Host copy (numpy, float64) of the current Wigner function."""
        if self._host_cache is None:
            self._host_cache = self._W.double().cpu().numpy()
        return self._host_cache

    def _returned_state(self):
        return self.wignerfunction

    def get_average(self, f):
        """<f(X, P)> = sum W f dXdP for a callable f(self, X, P) or f(X, P) (or a P x X array)."""
        if isinstance(f, FunctionType):
            try:
                F = f(self, self.X, self.P)
            except TypeError:
                F = f(self.X, self.P)
        elif callable(f):
            F = f(self.X, self.P)
        else:
            F = f
        return self._grid_average(np.asarray(F, dtype=np.float64))


class WignerBlochFFTW1D(WignerMoyalFTTW1D):
    """Gibbs state by split-operator propagation of the phase-space Bloch
    equation (drop-in for wigner_bloch_fftw_1d.py:6).  Reproduces the
    reference's FFTW exponents exp(-dbeta/2 (V- + V+ - min)) and
    exp(-dbeta (K+ + K- - min)) (:65-100), i.e. the state exp(-2H/kT)."""

    def __init__(self, **kwargs):
        try:
            self.kT = kwargs["kT"]
        except KeyError:
            raise AttributeError("Temperature (kT) was not specified") from None
        if self.kT > 0:
            self.dbeta = kwargs.get("dbeta", 0.01)
            self.num_beta_steps = 1.0 / (self.kT * self.dbeta)
            if round(self.num_beta_steps) != self.num_beta_steps:
                self.num_beta_steps = round(self.num_beta_steps)
                self.dbeta = 1.0 / (self.kT * self.num_beta_steps)
            self.num_beta_steps = int(self.num_beta_steps)
        else:
            raise NotImplementedError("The calculation of the ground state Wigner function has not been implemented")
        kwargs = dict(kwargs)
        kwargs.update(dbeta=self.dbeta, dt=self.dbeta)
        super().__init__(**kwargs)
        self.isEhrenfest = False
        self._tab_real = True
        h = self.hbar
        t = self.t
        ev = self._v_at(self._Xk - 0.5 * h * self._Tk, t) + self._v_at(self._Xk + 0.5 * h * self._Tk, t)
        ev = np.broadcast_to(ev, self.X_minus.shape)
        self._expV = np.exp(-self.dbeta * 0.5 * (ev - ev.min())) * self._abs
        ek = self._k_at(self._Pk + 0.5 * h * self._Lk, t) + self._k_at(self._Pk - 0.5 * h * self._Lk, t)
        ek = np.broadcast_to(ek, self.P_plus.shape)
        self._expK = np.exp(-self.dbeta * (ek - ek.min()))

    def _tables_static(self):
        return True

    def _static_tables(self):
        if getattr(self, "_tabV_dev", None) is None:
            self._tabV_dev = self._upload_table(self._expV, self.X_minus.shape)
            self._tabK_dev = self._upload_table(self._expK, self.P_plus.shape)
        return self._tabV_dev, self._tabK_dev

    def get_exp_v(self, t):
        return self._expV

    def get_exp_k(self, t):
        return self._expK

    def get_gibbs_state(self):
        """Start from W = const and take num_beta_steps Bloch steps (:102-109)."""
        self.set_wignerfunction(lambda _, x, p: 0 * x + 0 * p + 1.0)
        return self.propagate(self.num_beta_steps)


class WignerRandomCollisionModelFFTW1D(WignerMoyalFTTW1D):
    """Random-collision open-system dynamics dW/dt = {{H, W}} + gamma (W0 - W)
    (drop-in for wigner_random_collision_model_fftw_1d.py:6).  Each step runs
    blend -> Moyal step -> blend with the blends fused into the column passes."""

    def __init__(self, **kwargs):
        super().__init__(**kwargs)
        _require(self, "gamma", "Collision rate (gamma) was not specified")
        self.w_coeff = np.exp(-self.gamma * 0.5 * self.dt)
        gibbs = WignerBlochFFTW1D(**kwargs)
        self.scaled_gibbs_state = gibbs.get_gibbs_state() * (1 - self.w_coeff)
        del gibbs
        if self.isEhrenfest:
            dc = self.scaled_gibbs_state.sum(axis=0)
            dc = dc / dc.sum()
            self.X_average_gibbs = np.dot(dc, self.X.reshape(-1))
            dm = self.scaled_gibbs_state.sum(axis=1)
            dm = dm / dm.sum()
            self.P_average_gibbs = np.dot(dm, self.P.reshape(-1))
        self._step_kind = FW_STEP_SPLIT
        self._s0 = to_device(self.scaled_gibbs_state, self._rt, self.device)
        self._blend_c = float(self.w_coeff)

    def _ehrenfest_from_obs(self, obs):
        n = obs.shape[0]
        super()._ehrenfest_from_obs(obs)
        for k in range(len(self.X_average) - n, len(self.X_average)):
            self.X_average_RHS[k] += self.gamma * (self.X_average_gibbs - self.X_average[k])
            self.P_average_RHS[k] += self.gamma * (self.P_average_gibbs - self.P_average[k])

    def single_step_propagation(self):
        obs = self._propagate_chunk(1, self.t - self.dt)
        self._W.mul_(float(obs[0, 0]) * self.dXdP)
        self._host_cache = None
        return self.wignerfunction

    def get_Ehrenfest(self, t):
        r = super().get_Ehrenfest(t)
        if self.isEhrenfest:
            self.X_average_RHS[-1] += self.gamma * (self.X_average_gibbs - self.X_average[-1])
            self.P_average_RHS[-1] += self.gamma * (self.P_average_gibbs - self.P_average[-1])
        return r
