"""FP64 numpy restatement of the reference's density-matrix propagators.

TEST INFRASTRUCTURE ONLY -- the oracle for ``RhoVNeumannCUDA1D``
(rho_vneumann_cuda_1d.py) and ``RhoBlochCUDA1D`` (rho_bloch_cuda_1d.py).
These classes need PyCUDA + scikit-cuda + a GPU, so they cannot run here;
this file follows their kernel strings line by line instead:

* grids (:94-110): X = linspace(-A, A - dX, N); P = fftfreq(N, dX/2pi),
  dP = P[1] - P[0]; kernels index X = dX (j - N/2), P = dP ((j + N/2) % N - N/2);
  rho[i][j] = <X'_i| rho |X_j> (:676-679).
* step (:340-353): rho *= exp(-i dt/2 (V(X) - V(X'))) * abs_boundary_x (at t),
  2-D forward FFT, rho *= exp(-i dt (K(P) - K(P'))) * abs_boundary_p, 2-D
  unnormalised inverse FFT, expV again; propagate (:355-374): t += dt, step,
  rho /= trace(rho) dX (complex trace).
* observables (:431-472): successive x-multiplies and momentum multiplies
  (row FFT / N, multiply, row inverse FFT) on a copy, then Re trace * dX.
* purity (:474-488): sum |rho|^2 dX^2.
* Wigner transform (:502-592): shear X, shear Y, shear X (Larkin et al.),
  sign flip, inverse FFT along axis 0, sign flip, normalise by sum * wigner_dxdp.
* Bloch (rho_bloch_cuda_1d.py:69-241): exponents -dbeta/4 (V + V' - V_min),
  -dbeta/2 (K + K' - K_min) at t_initial with K_min = 0 (the reference's
  ``fill_K`` multiplies into a zeroed array, :364), delta initial state.
"""
from __future__ import annotations

import numpy as np


class RhoOracle:
    def __init__(self, *, X_gridDIM, X_amplitude, dt, V, K, t=0.0, diff_V=None, diff_K=None,
                 abs_boundary_x=None, abs_boundary_p=None):
        N = self.N = X_gridDIM
        self.dt, self.t = float(dt), float(t)
        self.V, self.K, self.diff_V, self.diff_K = V, K, diff_V, diff_K
        self.dX = 2.0 * X_amplitude / N
        self.X = np.linspace(-X_amplitude, X_amplitude - self.dX, N)
        self.P = np.fft.fftfreq(N, self.dX / (2 * np.pi))
        self.dP = self.P[1] - self.P[0]
        j = np.arange(N)
        self.Xk = self.dX * (j - 0.5 * N)                       # kernel X grid
        self.Pk = self.dP * ((j + N // 2) % N - 0.5 * N)         # kernel (fft-ordered) P grid
        self.P_wigner = np.fft.fftshift(self.P / np.sqrt(2.0))[:, np.newaxis]
        self.X_wigner = (self.X / np.sqrt(2.0))[np.newaxis, :]
        self.wigner_dxdp = (self.X[1] - self.X[0]) * (self.P[1] - self.P[0]) / 2.0
        self.bx = 1.0 if abs_boundary_x is None else abs_boundary_x(self.Xk[None, :], self.Xk[:, None])
        self.bp = 1.0 if abs_boundary_p is None else abs_boundary_p(self.Pk[None, :], self.Pk[:, None])
        self.isEhrenfest = diff_V is not None and diff_K is not None
        self.X_average, self.P_average, self.X_average_RHS, self.P_average_RHS = [], [], [], []
        self.hamiltonian_average = []
        self.rho = np.zeros((N, N), complex)
        self.mode = "vn"

    # time-dependent callables take (x, t)
    def _v(self, x, t):
        try:
            return self.V(x, t)
        except TypeError:
            return self.V(x)

    def _k(self, p, t):
        try:
            return self.K(p, t)
        except TypeError:
            return self.K(p)

    def set_rho(self, R):
        self.rho = np.array(R, dtype=complex)
        self.rho /= np.trace(self.rho) * self.dX
        return self

    def exp_v(self, t):
        if self.mode == "bloch":
            return self._bv
        v = self._v(self.Xk, t)
        return np.exp(-0.5j * self.dt * (v[None, :] - v[:, None])) * self.bx

    def exp_k(self, t):
        if self.mode == "bloch":
            return self._bk
        k = self._k(self.Pk, t)
        return np.exp(-1j * self.dt * (k[None, :] - k[:, None])) * self.bp

    def single_step(self):
        """rho_vneumann_cuda_1d.py:340-353 (cuFFT inverse unnormalised)."""
        ev = self.exp_v(self.t)
        r = self.rho * ev
        r = np.fft.fft2(r)
        r *= self.exp_k(self.t)
        r = np.fft.ifft2(r) * (self.N * self.N)
        self.rho = r * ev
        return self.rho

    def propagate(self, steps=1):
        for _ in range(steps):
            self.t += self.dt
            self.single_step()
            self.rho /= np.trace(self.rho) * self.dX
            self.get_Ehrenfest(self.t)
        return self.rho

    def get_average(self, observable, t=None):
        """Tr[rho O1 O2 ...] * dX with alternating x / p operators (:431-472)."""
        t = self.t if t is None else t
        tmp = self.rho.copy()
        is_x = False
        for obs in observable:
            is_x = not is_x
            if obs is None:
                continue
            if is_x:
                tmp = tmp * np.broadcast_to(obs(self.Xk, t), (self.N,))[None, :]
            else:
                tmp = np.fft.fft(tmp, axis=1) / self.N
                tmp = tmp * np.broadcast_to(obs(self.Pk, t), (self.N,))[None, :]
                tmp = np.fft.ifft(tmp, axis=1) * self.N
        return np.trace(tmp).real * self.dX

    def get_purity(self):
        return np.sum(np.abs(self.rho) ** 2) * self.dX ** 2

    def get_Ehrenfest(self, t):
        if not self.isEhrenfest:
            return
        self.X_average.append(self.get_average((lambda x, t: x,), t))
        self.X_average_RHS.append(self.get_average((None, self.diff_K), t))
        self.P_average.append(self.get_average((None, lambda p, t: p), t))
        self.P_average_RHS.append(-self.get_average((self.diff_V,), t))
        self.hamiltonian_average.append(self.get_average((None, self._k), t) + self.get_average((self._v,), t))

    def get_wignerfunction(self):
        """rho_vneumann_cuda_1d.py:502-592."""
        N = self.N
        Pj = self.Pk[None, :]
        Xpi = self.Xk[:, None]
        Xj = self.Xk[None, :]
        Ppi = self.Pk[:, None]
        a = np.tan(np.pi / 8.0)
        b = -np.sin(np.pi / 4.0)
        shx = np.exp(1j * (-a * Pj * Xpi))
        shy = np.exp(1j * (-b * Ppi * Xj))
        tmp = np.fft.ifft(np.fft.fft(self.rho, axis=1) * shx, axis=1)
        tmp = np.fft.ifft(np.fft.fft(tmp, axis=0) * shy, axis=0)
        tmp = np.fft.ifft(np.fft.fft(tmp, axis=1) * shx, axis=1)
        sign = (1 - 2 * (np.arange(N) % 2))[:, None]
        tmp = tmp * sign
        tmp = np.fft.ifft(tmp, axis=0) * N
        tmp = tmp * sign
        tmp /= tmp.sum() * self.wigner_dxdp
        return tmp

    def get_wigner_time(self, wigner_current, wigner_init, t, Ip, H):
        """rho_vneumann_cuda_1d.py:594-620, 842-857: H(x, p, t) on the Wigner grid."""
        N = self.N
        X = (self.dX * (np.arange(N) - 0.5 * N) / np.sqrt(2.0))[None, :]
        P = (self.dP * (np.arange(N) - 0.5 * N) / np.sqrt(2.0))[:, None]
        h = H(X, P, t)
        ind = 0.5 * (1 + np.signbit(h + Ip).astype(int))
        return np.sum(ind * (np.real(wigner_current) - wigner_init)) * self.wigner_dxdp

    # -- Bloch ------------------------------------------------------------------
    def setup_bloch(self, t_initial=0.0):
        """rho_bloch_cuda_1d.py:69-97 (V_min over V(X) + V(X'); K_min = 0)."""
        v = self._v(self.Xk, t_initial)
        k = self._k(self.Pk, t_initial)
        self._vsum = v[None, :] + v[:, None]
        self._ksum = k[None, :] + k[:, None]
        self.V_min = self._vsum.min()
        self.K_min = 0.0
        self.mode = "bloch"
        return self

    def bloch_single_step(self, dbeta):
        self._bv = np.exp(-0.25 * dbeta * (self._vsum - self.V_min))
        self._bk = np.exp(-0.5 * dbeta * (self._ksum - self.K_min))
        self.single_step()
        self.rho /= np.trace(self.rho) * self.dX
        return self.rho

    def get_ground_state(self, dbeta, abs_tol_purity=1e-12):
        """rho_bloch_cuda_1d.py:162-221: imaginary-time steps from the delta
        state, each accepted only if the purity stays <= 1 and the energy
        Tr[rho K] + Tr[rho V] decreased; otherwise the previous state is
        restored and dbeta halved."""
        prev_e = cur_e = np.inf
        prev_p = cur_p = 0.0
        self.set_rho(np.eye(self.N))
        prev = self.rho.copy()
        while cur_p < (1.0 - abs_tol_purity) and dbeta > 1e-12:
            self.bloch_single_step(dbeta)
            cur_p = self.get_purity()
            cur_e = self.get_average((None, self._k)) + self.get_average((self._v,))
            if cur_p <= 1.0 and cur_e < prev_e:
                prev_e, prev_p = cur_e, cur_p
                prev = self.rho.copy()
            else:
                self.rho = prev.copy()
                dbeta *= 0.5
                cur_e, cur_p = prev_e, prev_p
        return self.rho

    def get_gibbs_state(self, kT, dbeta):
        """rho_bloch_cuda_1d.py:124-160 (delta initial state)."""
        nb = 1.0 / (kT * dbeta)
        if round(nb) != nb:
            nb = round(nb)
            dbeta = 1.0 / (kT * nb)
        self.set_rho(np.eye(self.N))
        for _ in range(int(nb)):
            self.bloch_single_step(dbeta)
            if not self.get_purity() < 1.0:
                break
        return self.rho
