"""FP64 numpy restatement of the reference's Wigner-function propagators.

TEST INFRASTRUCTURE ONLY -- the oracle.  Imported by ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s ``cpu_baseline`` /
``--impl reference`` leg, never by the product package.  It restates, in
plain numpy (pocketfft, FP64), what the reference computes:

* ``WignerMoyalFTTW1D``  (wigner_moyal_fftw_1d.py:101-481) -- convention "fftw":
  numpy-style grids with a negative Nyquist entry in Theta/Lambda
  (:110-127), phases evaluated at the already-incremented time t (:402,:429),
  normalised inverse transforms (pyFFTW default), optional absorbing
  boundary from ``alpha`` (:135-156), marginal-based Ehrenfest (:442-481).
* ``WignerMoyalCUDA1D``  (wigner_moyal_cuda_1d.py:113-143, :564-664) --
  convention "cuda": Theta_i = dTheta*i, Lambda_j = dLambda*j (positive
  Nyquist, :598, :638), X_j = dX*(j - X/2) (:637), phases at t + dt/2
  (:602, :643), boundary factors abs_boundary_x_theta / abs_boundary_lambda_p
  in the exponents and abs_boundary_x_p after the step (:516-517),
  observables as sum W*f*dXdP (:378-396).
* ``WignerBlochFFTW1D`` (wigner_bloch_fftw_1d.py:22-109): exponents
  exp(-dbeta/2 (V- + V+ - min)) and exp(-dbeta (K+ + K- - min)) -- twice the
  CUDA class's, so the result is the Gibbs state of exp(-2H/kT).
* ``WignerBlochCUDA1D`` (wigner_bloch_cuda_1d.py:72-254): exponents
  -dbeta/4 (V- + V+ - V_min), -dbeta/2 (K+ + K- - K_min) at t_initial,
  purity guard, ground state with roll-back and dbeta halving.
* ``WignerRandomCollisionModelFFTW1D``
  (wigner_random_collision_model_fftw_1d.py:16-94): W <- c W + (1-c) W0 around
  every Moyal step, c = exp(-gamma dt/2), W0 the FFTW Bloch Gibbs state.

User potentials are Python callables here; time dependence is detected the
way the reference does it (call with one argument, TypeError -> time
dependent, wigner_moyal_fftw_1d.py:164-213).
"""
from __future__ import annotations

import numpy as np

try:  # multi-threaded FFTs for the timed CPU baseline (same pocketfft kernels)
    import scipy.fft as _sfft
except ImportError:  # pragma: no cover
    _sfft = None


def _is_time_dependent(f, arg) -> bool:
    try:
        f(arg)
        return False
    except TypeError:
        return True


class WignerOracle:
    """One Wigner-function propagator (Moyal / Bloch / collision) in FP64."""

    def __init__(self, *, X_gridDIM, X_amplitude, P_gridDIM, P_amplitude, dt, V, K, t=0.0,
                 convention="fftw", diff_V=None, diff_K=None, alpha=None,
                 abs_boundary_x_theta=None, abs_boundary_lambda_p=None, abs_boundary_x_p=None,
                 fft_workers=None):
        assert X_gridDIM % 2 == 0 and P_gridDIM % 2 == 0
        self.fft_workers = fft_workers
        self.conv = convention
        self.Xn, self.Pn = X_gridDIM, P_gridDIM
        self.dt, self.t = float(dt), float(t)
        self.V, self.K, self.diff_V, self.diff_K = V, K, diff_V, diff_K
        self.dX = 2.0 * X_amplitude / X_gridDIM
        self.dP = 2.0 * P_amplitude / P_gridDIM
        self.dXdP = self.dX * self.dP
        if convention == "fftw":
            # wigner_moyal_fftw_1d.py:102-127
            self.X = np.linspace(-X_amplitude, X_amplitude - self.dX, X_gridDIM)[np.newaxis, :]
            self.P = np.linspace(-P_amplitude, P_amplitude - self.dP, P_gridDIM)[:, np.newaxis]
            self.Lambda = np.fft.fftfreq(X_gridDIM, self.dX / (2 * np.pi))[: X_gridDIM // 2 + 1][np.newaxis, :]
            self.Theta = np.fft.fftfreq(P_gridDIM, self.dP / (2 * np.pi))[: P_gridDIM // 2 + 1][:, np.newaxis]
        else:
            # wigner_moyal_cuda_1d.py:113-140 grids; kernels use index formulas :598, :637-638
            lam = np.fft.fftfreq(X_gridDIM, self.dX / (2 * np.pi))
            th = np.fft.fftfreq(P_gridDIM, self.dP / (2 * np.pi))
            dLambda, dTheta = lam[1] - lam[0], th[1] - th[0]
            self.X = (self.dX * (np.arange(X_gridDIM) - 0.5 * X_gridDIM))[np.newaxis, :]
            self.P = (self.dP * (np.arange(P_gridDIM) - 0.5 * P_gridDIM))[:, np.newaxis]
            self.Lambda = (dLambda * np.arange(X_gridDIM // 2 + 1))[np.newaxis, :]
            self.Theta = (dTheta * np.arange(P_gridDIM // 2 + 1))[:, np.newaxis]
        self.X_minus = self.X - 0.5 * self.Theta
        self.X_plus = self.X + 0.5 * self.Theta
        self.P_minus = self.P - 0.5 * self.Lambda
        self.P_plus = self.P + 0.5 * self.Lambda
        # absorbing boundaries
        self.alpha = alpha
        self.abs_boundary = self._abs_boundary(self.dt)
        self.b_x_theta = 1.0 if abs_boundary_x_theta is None else abs_boundary_x_theta(self.X, self.Theta)
        self.b_lambda_p = 1.0 if abs_boundary_lambda_p is None else abs_boundary_lambda_p(self.Lambda, self.P)
        self.b_x_p = None if abs_boundary_x_p is None else abs_boundary_x_p(self.X, self.P)
        self.V_td = _is_time_dependent(V, self.X_minus)
        self.K_td = _is_time_dependent(K, self.P_plus)
        self.mode = "moyal"
        self.isEhrenfest = diff_V is not None and diff_K is not None
        self.X_average, self.P_average = [], []
        self.X_average_RHS, self.P_average_RHS = [], []
        self.hamiltonian_average = []
        self.W = np.zeros((P_gridDIM, X_gridDIM))
        self.gamma = None

    def _abs_boundary(self, dt):
        """wigner_moyal_fftw_1d.py:139-156 (1 when alpha is not given)."""
        if self.alpha is None:
            return 1.0
        xmin = min(self.X_minus.min(), self.X_plus.min())
        xmax = max(self.X_minus.max(), self.X_plus.max())
        b = np.sin(np.pi * (self.X_plus - xmin) / (xmax - xmin))
        b = b * np.sin(np.pi * (self.X_minus - xmin) / (xmax - xmin))
        return np.abs(b) ** abs(self.alpha * dt)

    # -- potentials at time t (with one-argument fallback as in the reference)
    def _v(self, x, t):
        return self.V(x, t) if self.V_td else self.V(x)

    def _k(self, p, t):
        return self.K(p, t) if self.K_td else self.K(p)

    def _tphase(self):
        return self.t + 0.5 * self.dt if self.conv == "cuda" else self.t

    # -- exponents (wigner_moyal_fftw_1d.py:164-213; wigner_moyal_cuda_1d.py:592-663)
    def exp_v(self):
        if getattr(self, "_cache_v", None) is not None:
            return self._cache_v
        if self.mode == "bloch_fftw":
            return self._bloch_v
        if self.mode == "bloch_cuda":
            return self._bloch_v
        t = self._tphase()
        e = np.exp(-self.dt * 0.5j * (self._v(self.X_minus, t) - self._v(self.X_plus, t)))
        return e * self.abs_boundary * self.b_x_theta

    def exp_k(self):
        if getattr(self, "_cache_k", None) is not None:
            return self._cache_k
        if self.mode in ("bloch_fftw", "bloch_cuda"):
            return self._bloch_k
        t = self._tphase()
        e = np.exp(-self.dt * 1j * (self._k(self.P_plus, t) - self._k(self.P_minus, t)))
        return e * self.b_lambda_p

    def set_wignerfunction(self, W):
        W = np.asarray(W, dtype=np.float64)
        self.W = W.copy()
        self.W /= self.W.sum() * self.dXdP
        return self

    def single_step(self):
        """V/2 -> K -> V/2 (wigner_moyal_fftw_1d.py:397-416)."""
        ev, ek = self.exp_v(), self.exp_k()
        W = self.W
        if self.fft_workers and _sfft is not None:
            w = self.fft_workers
            rf = lambda a, ax: _sfft.rfft(a, axis=ax, workers=w)
            irf = lambda a, n, ax: _sfft.irfft(a, n=n, axis=ax, workers=w)
        else:
            rf = lambda a, ax: np.fft.rfft(a, axis=ax)
            irf = lambda a, n, ax: np.fft.irfft(a, n=n, axis=ax)
        W = irf(rf(W, 0) * ev, self.Pn, 0)
        W = irf(rf(W, 1) * ek, self.Xn, 1)
        W = irf(rf(W, 0) * ev, self.Pn, 0)
        if self.b_x_p is not None:  # wigner_moyal_cuda_1d.py:516-517
            W = W * self.b_x_p
        self.W = W

    def propagate(self, steps=1):
        """wigner_moyal_fftw_1d.py:418-440 (and the collision blend :56-76)."""
        for _ in range(steps):
            self.t += self.dt
            if self.gamma is not None:
                self.W = self.W * self.w_coeff + self.scaled_gibbs_state
            self.single_step()
            if self.gamma is not None:
                self.W = self.W * self.w_coeff + self.scaled_gibbs_state
            self.W /= self.W.sum() * self.dXdP
            self.get_Ehrenfest(self.t)
        return self.W

    def get_Ehrenfest(self, t):
        """wigner_moyal_fftw_1d.py:442-481 (+ collision amendment :78-94)."""
        if not self.isEhrenfest:
            return
        W = self.W
        dc = W.sum(axis=0)
        dc = dc / dc.sum()
        dm = W.sum(axis=1)
        dm = dm / dm.sum()
        dV = self.diff_V(self.X, t) if _is_time_dependent(self.diff_V, self.X) else self.diff_V(self.X)
        dK = self.diff_K(self.P, t) if _is_time_dependent(self.diff_K, self.P) else self.diff_K(self.P)
        self.X_average.append(np.dot(dc, self.X.reshape(-1)))
        self.P_average_RHS.append(-np.dot(dc, np.broadcast_to(dV, self.X.shape).reshape(-1)))
        self.P_average.append(np.dot(dm, self.P.reshape(-1)))
        self.X_average_RHS.append(np.dot(dm, np.broadcast_to(dK, self.P.shape).reshape(-1)))
        self.hamiltonian_average.append(
            np.dot(dm, np.broadcast_to(self._k(self.P, t), self.P.shape).reshape(-1))
            + np.dot(dc, np.broadcast_to(self._v(self.X, t), self.X.shape).reshape(-1)))
        if self.gamma is not None:
            self.X_average_RHS[-1] += self.gamma * (self.X_average_gibbs - self.X_average[-1])
            self.P_average_RHS[-1] += self.gamma * (self.P_average_gibbs - self.P_average[-1])

    def get_purity(self):
        return 2.0 * np.pi * np.sum(self.W ** 2) * self.dXdP

    def cache_exponents(self):
        """Freeze the current exponents (what the reference does for a
        time-independent Hamiltonian, wigner_moyal_fftw_1d.py:164-199)."""
        self._cache_v, self._cache_k = None, None
        self._cache_v, self._cache_k = self.exp_v(), self.exp_k()
        return self

    def get_average(self, f):
        return np.sum(self.W * f(self.X, self.P)) * self.dXdP

    # -- Bloch ----------------------------------------------------------------
    def setup_bloch_fftw(self, kT, dbeta=0.01):
        """wigner_bloch_fftw_1d.py:22-100 (exponents computed at self.t)."""
        nb = 1.0 / (kT * dbeta)
        if round(nb) != nb:
            nb = round(nb)
            dbeta = 1.0 / (kT * nb)
        self.num_beta_steps = int(nb)
        self.dbeta = self.dt = dbeta
        self.abs_boundary = self._abs_boundary(dbeta)  # the Bloch class is built with dt = dbeta
        t = self.t
        ev = self._v(self.X - 0.5 * self.Theta, t) + self._v(self.X + 0.5 * self.Theta, t)
        ev = np.exp(-dbeta * 0.5 * (ev - ev.min())) * self.abs_boundary
        ek = self._k(self.P + 0.5 * self.Lambda, t) + self._k(self.P - 0.5 * self.Lambda, t)
        ek = np.exp(-dbeta * (ek - ek.min()))
        self._bloch_v, self._bloch_k = ev, ek
        self.mode = "bloch_fftw"
        self.isEhrenfest = False
        return self

    def get_gibbs_state_fftw(self):
        """wigner_bloch_fftw_1d.py:102-109."""
        self.set_wignerfunction(np.ones((self.Pn, self.Xn)))
        return self.propagate(self.num_beta_steps)

    @staticmethod
    def get_dbeta_num_beta_steps(kT, dbeta):
        """wigner_bloch_cuda_1d.py:104-127."""
        if kT > 0:
            nb = 1.0 / (kT * dbeta)
            if round(nb) != nb:
                nb = round(nb)
                dbeta = 1.0 / (kT * nb)
            return dbeta, int(nb)
        return dbeta, np.inf

    def setup_bloch_cuda(self, t_initial=0.0):
        """wigner_bloch_cuda_1d.py:72-102 (V_min, K_min over the same grids)."""
        vs = self._v(self.X - 0.5 * self.Theta, t_initial) + self._v(self.X + 0.5 * self.Theta, t_initial)
        ks = self._k(self.P + 0.5 * self.Lambda, t_initial) + self._k(self.P - 0.5 * self.Lambda, t_initial)
        self._vs, self._ks = np.broadcast_to(vs, self.X_minus.shape), np.broadcast_to(ks, self.P_plus.shape)
        self.V_min, self.K_min = self._vs.min(), self._ks.min()
        self.mode = "bloch_cuda"
        return self

    def bloch_single_step(self, dbeta):
        """wigner_bloch_cuda_1d.py:229-254 (normalised at the end)."""
        self._bloch_v = np.exp(-0.25 * dbeta * (self._vs - self.V_min))
        self._bloch_k = np.exp(-0.5 * dbeta * (self._ks - self.K_min))
        self.single_step()
        self.W /= self.W.sum() * self.dXdP
        return self.W

    def get_gibbs_state_cuda(self, kT, dbeta):
        """wigner_bloch_cuda_1d.py:129-165."""
        dbeta, n = self.get_dbeta_num_beta_steps(kT, dbeta)
        self.set_wignerfunction(np.full((self.Pn, self.Xn), 1.0 / (self.Pn * self.Xn)))
        self.bloch_stopped_at = None
        for k in range(n):
            self.bloch_single_step(dbeta)
            if not self.get_purity() < 1.0:
                self.bloch_stopped_at = k
                break
        return self.W

    def get_ground_state_cuda(self, dbeta, abs_tol_purity=1e-12):
        """wigner_bloch_cuda_1d.py:167-227: imaginary-time steps from W = const,
        each accepted only if purity <= 1, the energy <K> + <V> decreased and
        sigma_x sigma_p >= 1/2; otherwise the previous state is restored and
        dbeta halved.  Observables on the kernel grids (CUDA convention)."""
        prev_e = cur_e = np.inf
        prev_p = cur_p = 0.0
        self.set_wignerfunction(np.full((self.Pn, self.Xn), 1.0 / (self.Pn * self.Xn)))
        prev_W = self.W.copy()
        X, P = self.X, self.P
        t = self.t
        while cur_p < (1.0 - abs_tol_purity) and dbeta > 1e-12:
            self.bloch_single_step(dbeta)
            cur_p = self.get_purity()
            av = lambda F: np.sum(self.W * F) * self.dXdP  # noqa: E731
            cur_e = av(np.broadcast_to(self._k(P, t), self.W.shape)) + av(np.broadcast_to(self._v(X, t), self.W.shape))
            sig = np.sqrt((av(X * X + 0 * P) - av(X + 0 * P) ** 2) * (av(P * P + 0 * X) - av(P + 0 * X) ** 2))
            if cur_p <= 1.0 and cur_e < prev_e and sig >= 0.5:
                prev_e, prev_p = cur_e, cur_p
                prev_W = self.W.copy()
            else:
                self.W = prev_W.copy()
                dbeta *= 0.5
                cur_e, cur_p = prev_e, prev_p
        return self.W

    # -- random collision ------------------------------------------------------
    def setup_collision(self, gamma, kT, dbeta=0.01):
        """wigner_random_collision_model_fftw_1d.py:16-54 (W0 from the FFTW Bloch class)."""
        self.gamma = float(gamma)
        self.w_coeff = np.exp(-self.gamma * 0.5 * self.dt)
        b = WignerOracle(X_gridDIM=self.Xn, X_amplitude=self.Xn * self.dX / 2, P_gridDIM=self.Pn,
                         P_amplitude=self.Pn * self.dP / 2, dt=self.dt, V=self.V, K=self.K, t=self.t,
                         convention="fftw", alpha=self.alpha)
        b.setup_bloch_fftw(kT, dbeta)
        g = b.get_gibbs_state_fftw().copy()
        self.gibbs_state = g.copy()
        self.scaled_gibbs_state = g * (1.0 - self.w_coeff)
        if self.isEhrenfest:
            dc = self.scaled_gibbs_state.sum(axis=0)
            dc = dc / dc.sum()
            self.X_average_gibbs = np.dot(dc, self.X.reshape(-1))
            dm = self.scaled_gibbs_state.sum(axis=1)
            dm = dm / dm.sum()
            self.P_average_gibbs = np.dot(dm, self.P.reshape(-1))
        return self


def exact_harmonic_gibbs(omega, kT, X, P):
    """Exact Gibbs Wigner function of H = (p^2 + omega^2 x^2)/2 at temperature kT
    (wigner_bloch_fftw_1d.py:152-154)."""
    th = np.tanh(0.5 * omega / kT)
    return th / np.pi * np.exp(-2.0 * th * (0.5 * P ** 2 + 0.5 * omega ** 2 * X ** 2) / omega)
