"""Drop-ins for the reference's CUDA-string Wigner classes.

* ``WignerMoyalCUDA1D`` -- wigner_moyal_cuda_1d.py:10
* ``WignerBlochCUDA1D`` -- wigner_bloch_cuda_1d.py:8

V, K, diff_V, diff_K, the absorbing boundaries, initial states and
observables are C-expression strings as in the reference; they are compiled
once per instance with NVRTC (``cexpr.ExprModule``) in the reference's
environment (every numeric keyword as a ``const``, ``consts`` and
``functions`` appended) and tabulated in FP64 on the device.  Grids follow
the reference kernels' index formulas: X_j = dX (j - X/2), P_i = dP (i - P/2),
Theta_i = dTheta i, Lambda_j = dLambda j (positive Nyquist entries), and the
exponents of the step ending at t are evaluated at t + dt/2
(wigner_moyal_cuda_1d.py:592-663).  The cuFFT inverses of the reference are
unnormalised; after the per-step renormalisation this makes no difference,
and ``single_step_propagation`` reproduces the P*X*P factor.
"""
from __future__ import annotations

from types import FunctionType

import numpy as np
import torch

from . import cexpr
from ._device import DeviceArray, to_device
from .wigner import _WignerBase, _require

_T_PROBE = (0.0, 1.2345678)


class WignerMoyalCUDA1D(_WignerBase):
    """Second-order split-operator Moyal propagator with C-string Hamiltonians
    (drop-in for wigner_moyal_cuda_1d.py:10)."""

    _conv = "cuda"

    def __init__(self, **kwargs):
        super().__init__(**kwargs)
        for name in ("V", "K"):
            if not isinstance(getattr(self, name), str):
                raise TypeError(f"{name} must be a string of C code (use WignerMoyalFTTW1D for Python callables)")
        kw = {k: v for k, v in kwargs.items() if k != "t"}
        kw.update(dX=self.dX, dP=self.dP, dLambda=self.dLambda, dTheta=self.dTheta)
        self.cuda_consts = cexpr.cuda_consts(kw, user_consts=getattr(self, "consts", ""))
        self.functions = getattr(self, "functions", "")
        try:
            self.abs_boundary_x_theta
        except AttributeError:
            self.abs_boundary_x_theta = "1."
        try:
            self.abs_boundary_lambda_p
        except AttributeError:
            self.abs_boundary_lambda_p = "1."
        self.hamiltonian = self.K + " + " + self.V
        exprs = {"fw_V": "V(X, t)", "fw_K": "K(P, t)", "fw_bxt": self.abs_boundary_x_theta,
                 "fw_blp": self.abs_boundary_lambda_p}
        try:
            self.diff_K
            self.diff_V
            self.isEhrenfest = True
            exprs.update(fw_dV=self.diff_V, fw_dK=self.diff_K)
        except AttributeError:
            self.isEhrenfest = False
        bxp = getattr(self, "abs_boundary_x_p", None)
        if bxp is not None:
            exprs["fw_bxp"] = bxp
        self._extra_exprs(exprs)
        self._mod = cexpr.ExprModule(self.cuda_consts, self.functions, exprs, K=self.K, V=self.V)
        self._observables = {}
        # time dependence of the strings (the reference re-evaluates them at every step anyway)
        self._v_td = self._probe_td("fw_V", X=self._Xk)
        self._k_td = self._probe_td("fw_K", P=self._Pk)
        # boundary factors at the initial time
        self._bxt = self._mod.eval_grid("fw_bxt", self.X_minus.shape, X=self._Xk, Theta=self._Tk, t=self.t,
                                        i=np.arange(self.P_gridDIM // 2 + 1)[:, None],
                                        j=np.arange(self.X_gridDIM)[None, :])
        self._blp = self._mod.eval_grid("fw_blp", self.P_plus.shape, Lambda=self._Lk, P=self._Pk, t=self.t,
                                        i=np.arange(self.P_gridDIM)[:, None],
                                        j=np.arange(self.X_gridDIM // 2 + 1)[None, :])
        if bxp is not None:
            b = self._mod.eval_grid("fw_bxp", self._W.shape, X=self._Xk, P=self._Pk, t=self.t)
            self._bxp = to_device(b, self._rt, self.device)
        if self.isEhrenfest:
            self.X_average, self.P_average = [], []
            self.X_average_RHS, self.P_average_RHS = [], []
            self.hamiltonian_average = []
            self._w_td = self._v_td or self._k_td or self._probe_td("fw_dV", X=self._Xk) or \
                self._probe_td("fw_dK", P=self._Pk)
            self._w_static = None

    def _extra_exprs(self, exprs):
        pass

    def _probe_td(self, name, **coords):
        key = next(iter(coords))
        a = self._mod.eval_grid(name, np.shape(coords[key]), t=_T_PROBE[0], **coords)
        b = self._mod.eval_grid(name, np.shape(coords[key]), t=_T_PROBE[1], **coords)
        return not np.array_equal(a, b)

    # -- hooks ----------------------------------------------------------------
    def _v_at(self, x, t):
        return self._mod.eval_grid("fw_V", np.shape(x), X=x, t=t)

    def _k_at(self, p, t):
        return self._mod.eval_grid("fw_K", np.shape(p), P=p, t=t)

    def _v_time_dependent(self):
        return self._v_td

    def _k_time_dependent(self):
        return self._k_td

    def _b_x_theta(self):
        return self._bxt

    def _b_lambda_p(self):
        return self._blp

    def _unnormalised_factor(self):
        return float(self.P_gridDIM) * self.X_gridDIM * self.P_gridDIM

    # -- observables ----------------------------------------------------------
    def _weights_at(self, t):
        X, P = self._Xk.reshape(-1), self._Pk.reshape(-1)
        wx = torch.stack([torch.as_tensor(X, device=self.device),
                          self._mod.eval("fw_dV", X.size, X=X, t=t),
                          self._mod.eval("fw_V", X.size, X=X, t=t)])
        wp = torch.stack([torch.as_tensor(P, device=self.device),
                          self._mod.eval("fw_dK", P.size, P=P, t=t),
                          self._mod.eval("fw_K", P.size, P=P, t=t)])
        return wx.contiguous(), wp.contiguous()

    def _obs_weights(self, times):
        if not self.isEhrenfest:
            return None, None
        if not self._w_td:
            if self._w_static is None:
                self._w_static = self._weights_at(self.t)
            return self._w_static
        pairs = [self._weights_at(t) for t in times]
        return torch.stack([a for a, _ in pairs]).contiguous(), torch.stack([b for _, b in pairs]).contiguous()

    def get_Ehrenfest(self, t):
        """Append the Ehrenfest observables of the current state at time t
        (wigner_moyal_cuda_1d.py:542-562)."""
        if self.isEhrenfest:
            self.X_average.append(self.get_average("X"))
            self.X_average_RHS.append(self.get_average(self.diff_K))
            self.P_average.append(self.get_average("P"))
            self.P_average_RHS.append(-self.get_average(self.diff_V))
            self.hamiltonian_average.append(self.get_average(self.hamiltonian))

    def get_average(self, observable):
        """<observable(X, P, t)> = sum W f dXdP for a C-expression string
        (wigner_moyal_cuda_1d.py:378-396); compiled once per string."""
        if not isinstance(observable, str):
            raise TypeError("observable must be a string of C code")
        mod = self._observables.get(observable)
        if mod is None:
            mod = self._observables[observable] = cexpr.ExprModule(self.cuda_consts, self.functions,
                                                                   {"fw_obs": observable}, K=self.K, V=self.V)
        n = self._W.numel()
        i = np.repeat(np.arange(self.P_gridDIM), self.X_gridDIM)
        j = np.tile(np.arange(self.X_gridDIM), self.P_gridDIM)
        F = mod.eval("fw_obs", n, X=self.dX * (j - 0.5 * self.X_gridDIM), P=self.dP * (i - 0.5 * self.P_gridDIM),
                     t=self.t, i=i, j=j, indexTotal=j + i * self.X_gridDIM)
        return self._grid_average_dev(F.view(self._W.shape))

    def _grid_average_dev(self, F):
        from ._device import ptr, stream_handle
        from ._lib import check
        out = torch.empty(2, dtype=torch.float64, device=self.device)
        check(self._lib.fw_wigner_weighted_sum(self._plan, ptr(self._W), self._W.numel(), ptr(F.contiguous()),
                                               ptr(out), stream_handle()), "fw_wigner_weighted_sum")
        return float(out[0]) * self.dXdP

    def get_sigma_x_sigma_p(self):
        return np.sqrt((self.get_average("X * X") - self.get_average("X") ** 2)
                       * (self.get_average("P * P") - self.get_average("P") ** 2))

    # -- state ----------------------------------------------------------------
    def set_wignerfunction(self, new_wigner_func):
        """Array (numpy / torch / DeviceArray), F(self, X, P), a C string of X
        and P, or a float; then normalise (wigner_moyal_cuda_1d.py:454-494)."""
        if isinstance(new_wigner_func, (np.ndarray, torch.Tensor, DeviceArray)):
            self._set_state_array(new_wigner_func)
        elif isinstance(new_wigner_func, FunctionType):
            val = new_wigner_func(self, self.X, self.P)
            self._set_state_array(np.broadcast_to(np.asarray(val, dtype=np.float64), self._W.shape))
        elif isinstance(new_wigner_func, str):
            mod = cexpr.ExprModule(self.cuda_consts, self.functions, {"fw_init": new_wigner_func})
            n = self._W.numel()
            i = np.repeat(np.arange(self.P_gridDIM), self.X_gridDIM)
            j = np.tile(np.arange(self.X_gridDIM), self.P_gridDIM)
            W = mod.eval("fw_init", n, X=self.dX * (j - 0.5 * self.X_gridDIM),
                         P=self.dP * (i - 0.5 * self.P_gridDIM), i=i, j=j, indexTotal=j + i * self.X_gridDIM)
            self._W.copy_(W.view(self._W.shape).to(self._rt))
        elif isinstance(new_wigner_func, float):
            self._W.fill_(new_wigner_func)
        else:
            raise NotImplementedError("new_wigner_func must be either function or numpy.array")
        self._normalise_()
        return self

    @property
    def wignerfunction(self) -> DeviceArray:
        return DeviceArray(self._W)

    def _returned_state(self):
        return DeviceArray(self._W)


class WignerBlochCUDA1D(WignerMoyalCUDA1D):
    """Gibbs and ground states by the phase-space Bloch equation with
    C-string Hamiltonians (drop-in for wigner_bloch_cuda_1d.py:8).  Exponents
    -dbeta/4 (V- + V+ - V_min) and -dbeta/2 (K+ + K- - K_min) at t_initial
    (:290-359)."""

    def __init__(self, **kwargs):
        kwargs = dict(kwargs)
        if "t_initial" not in kwargs:
            kwargs.update(t_initial=0.0)
            print("Warning: Initial time (t_initial) was not specified. So the default value was used t_initial = 0.")
        self.kT = kwargs.pop("kT", 0.0)
        self.dbeta = kwargs.pop("dbeta", 0.01)
        if "dt" not in kwargs:
            kwargs.update(dt=self.dbeta)
        super().__init__(**kwargs)
        h = self.hbar
        ti = float(self.t_initial)
        vs = self._v_at(self._Xk - 0.5 * h * self._Tk, ti) + self._v_at(self._Xk + 0.5 * h * self._Tk, ti)
        ks = self._k_at(self._Pk + 0.5 * h * self._Lk, ti) + self._k_at(self._Pk - 0.5 * h * self._Lk, ti)
        self._vsum = np.broadcast_to(vs, self.X_minus.shape)
        self._ksum = np.broadcast_to(ks, self.P_plus.shape)
        self.V_min = float(self._vsum.min())
        self.K_min = float(self._ksum.min())
        self.cuda_consts += "    const double V_min = %.15e;\n" % self.V_min
        self.cuda_consts += "    const double K_min = %.15e;\n" % self.K_min
        self._bloch_cache = {}
        # per-step monitors: sum W, sum W^2, <x>, <x^2>, <V>, <p>, <p^2>, <K>
        X, P = self._Xk.reshape(-1), self._Pk.reshape(-1)
        self._bw = (to_device(np.stack([X, X * X, self._v_at(self._Xk, ti).reshape(-1)]), torch.float64, self.device),
                    to_device(np.stack([P, P * P, self._k_at(self._Pk, ti).reshape(-1)]), torch.float64, self.device))

    def get_V_min(self):
        return self.V_min

    def get_K_min(self):
        return self.K_min

    @classmethod
    def get_dbeta_num_beta_steps(cls, kT, dbeta):
        """wigner_bloch_cuda_1d.py:104-127."""
        if kT > 0:
            num_beta_steps = 1.0 / (kT * dbeta)
            if round(num_beta_steps) != num_beta_steps:
                num_beta_steps = round(num_beta_steps)
                dbeta = 1.0 / (kT * num_beta_steps)
            num_beta_steps = int(num_beta_steps)
        else:
            num_beta_steps = np.inf
        return dbeta, num_beta_steps

    def _bloch_tables(self, dbeta):
        key = float(dbeta)
        tabs = self._bloch_cache.get(key)
        if tabs is None:
            ev = np.exp(-0.25 * dbeta * (self._vsum - self.V_min))
            ek = np.exp(-0.5 * dbeta * (self._ksum - self.K_min))
            tabs = (self._upload_table(ev, self.X_minus.shape, real=True), 0,
                    self._upload_table(ek, self.P_plus.shape, real=True), 0, True)
            if len(self._bloch_cache) > 8:
                self._bloch_cache.clear()
            self._bloch_cache[key] = tabs
        return tabs

    def _bloch_steps(self, dbeta, n):
        return self._propagate_chunk(n, self.t, tables=self._bloch_tables(dbeta), weights=self._bw)

    def _purity_from_obs(self, obs):
        S, S2 = obs[:, 0], obs[:, 1]
        return 2.0 * np.pi * self.hbar * S2 / (S * S * self.dXdP)

    def bloch_single_step_propagation(self, dbeta):
        """One Bloch step, normalised (wigner_bloch_cuda_1d.py:229-254)."""
        self._bloch_steps(float(dbeta), 1)
        return self.wignerfunction

    def get_gibbs_state(self, kT=None, dbeta=None, chunk=256):
        """Boltzmann-Gibbs state from W = const (wigner_bloch_cuda_1d.py:129-165):
        the step loop stops after the first step whose purity is >= 1."""
        dbeta = self.dbeta if dbeta is None else dbeta
        kT = self.kT if kT is None else kT
        dbeta, n = self.get_dbeta_num_beta_steps(kT, dbeta)
        dbeta = float(dbeta)
        self.set_wignerfunction(1.0 / float(self.P_gridDIM * self.X_gridDIM))
        done = 0
        while done < n:
            m = int(min(chunk, n - done))
            snap = self._W.clone()
            obs = self._bloch_steps(dbeta, m)
            bad = np.nonzero(~(self._purity_from_obs(obs) < 1.0))[0]
            if bad.size:
                k = int(bad[0])
                self._W.copy_(snap)
                obs = self._bloch_steps(dbeta, k + 1)
                kk = done + k
                print("Warning: Gibbs state calculations interupted because purity = %.10f > 1."
                      "Current kT = %.6f" % (self.get_purity(), 1 / (kk * dbeta) if kk else np.inf))
                break
            done += m
        return self.wignerfunction

    def get_ground_state(self, dbeta=None, abs_tol_purity=1e-12):
        """Ground state by imaginary-time steps with the reference's acceptance
        tests and roll-back / step halving (wigner_bloch_cuda_1d.py:167-227)."""
        previous_energy = current_energy = np.inf
        previous_purity = current_purity = 0.0
        dbeta = float(self.dbeta if dbeta is None else dbeta)
        self.set_wignerfunction(1.0 / float(self.P_gridDIM * self.X_gridDIM))
        previous = self._W.clone()
        while current_purity < (1.0 - abs_tol_purity) and dbeta > 1e-12:
            obs = self._bloch_steps(dbeta, 1)[0]
            S = obs[0]
            current_purity = float(self._purity_from_obs(obs[None, :])[0])
            xm, x2, vm, pm, p2, km = obs[2] / S, obs[3] / S, obs[4] / S, obs[5] / S, obs[6] / S, obs[7] / S
            current_energy = km + vm
            sigma = np.sqrt(max(x2 - xm * xm, 0.0) * max(p2 - pm * pm, 0.0))
            if current_purity <= 1.0 and current_energy < previous_energy and sigma >= 0.5:
                previous_energy, previous_purity = current_energy, current_purity
                previous.copy_(self._W)
                print("Current energy: %.5f; purity: 1 - %.2e; dbeta: %.2e" % (current_energy, 1 - current_purity, dbeta))
            else:
                self._W.copy_(previous)
                dbeta *= 0.5
                current_energy, current_purity = previous_energy, previous_purity
        self._host_cache = None
        return self.wignerfunction
