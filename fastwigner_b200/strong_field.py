"""Strong-field phase-space dynamics: a Wigner function driven by a laser field,
optionally with random-collision dephasing.

The reference expresses this as scripts, not a class:
strong_field_physics_fftw_1d.py:35-90 (velocity gauge, K = (p + A(t))^2 / 2,
Mathieu lattice, Gibbs initial state) and strong_field_physics_cuda_1d.py:24-82
(length gauge, V = V0(x) + x E(t)).  ``StrongFieldWigner`` runs either gauge
with the field split off the static Hamiltonian:

* velocity gauge: K(p + hbar l/2) - K(p - hbar l/2) = hbar l (p + A(t)), so the
  kinetic exponent is a static table exp(-i dt l p) times the per-step vector
  exp(-i dt A(t) l) over lambda;
* length gauge: V(x -/+ hbar th/2) differ by -hbar th E(t), so the potential
  exponent is the static V0 table times exp(i dt E(t) th / 2) over theta.

The per-step vectors are built in FP64 (A(t) from the user's closed form or
by Gauss-Legendre integration of E(t) in FP64) and applied inside the fused
passes; the bulk stays in the state precision.  Conventions (exponents at the
incremented time t, normalisation, Ehrenfest lists) are
WignerMoyalFTTW1D's; with ``gamma`` the step is the random-collision model's
blend -> Moyal step -> blend (wigner_random_collision_model_fftw_1d.py:56-76)
with W0 the Gibbs state at ``kT`` of the Hamiltonian at the initial time, field
included -- what the reference's Bloch class does with a time-dependent
Hamiltonian (wigner_bloch_fftw_1d.py:65-72, 86-93).
"""
from __future__ import annotations

import numpy as np
import torch

from ._device import to_device
from ._lib import FW_STEP_SPLIT
from .wigner import WignerBlochFFTW1D, WignerMoyalFTTW1D

_GL_X, _GL_W = np.polynomial.legendre.leggauss(8)


def integrate_field(E, t0, t1, pieces=4):
    """int_{t0}^{t1} E(t) dt in FP64 (composite 8-point Gauss-Legendre)."""
    edges = np.linspace(t0, t1, pieces + 1)
    tot = 0.0
    for a, b in zip(edges[:-1], edges[1:]):
        m, h = 0.5 * (a + b), 0.5 * (b - a)
        tot += h * np.sum(_GL_W * np.asarray(E(m + h * _GL_X), dtype=np.float64))
    return float(tot)


def integrate_intervals(E, t0s, t1s, pieces):
    """integrate_field(E, t0s[i], t1s[i], pieces) for every i, with E evaluated
    on all quadrature nodes of all intervals in one call (same rule, same
    order of operations); falls back to one call per interval when E does
    not take arrays of any shape."""
    t0s = np.asarray(t0s, dtype=np.float64)
    t1s = np.asarray(t1s, dtype=np.float64)
    edges = np.linspace(t0s, t1s, pieces + 1)             # (pieces + 1) x n
    a, b = edges[:-1], edges[1:]
    m, h = 0.5 * (a + b), 0.5 * (b - a)
    nodes = m[..., None] + h[..., None] * _GL_X            # pieces x n x 8
    try:
        vals = np.asarray(E(nodes), dtype=np.float64)
        if vals.shape != nodes.shape:
            raise ValueError
    except Exception:
        return np.array([integrate_field(E, x, y, pieces) for x, y in zip(t0s, t1s)])
    tot = np.zeros(t0s.shape)
    for c in range(pieces):
        tot += h[c] * np.sum(_GL_W * vals[c], axis=-1)
    return tot


def _on_times(f, times):
    """float(f(t)) for every t: one call on the array when f vectorises."""
    try:
        v = np.asarray(f(times), dtype=np.float64)
        if v.shape == times.shape:
            return v
    except Exception:
        pass
    return np.array([float(f(t)) for t in times])


class StrongFieldWigner(WignerMoyalFTTW1D):
    """Keywords: the WignerMoyalFTTW1D grid keywords, ``V`` (static V0(self, x)),
    ``gauge`` ("velocity" or "length"), the field as ``A(self, t)`` (velocity)
    and/or ``E(self, t)``; optional ``diff_V`` (of V0), ``gamma`` and ``kT`` (collision
    model), ``dbeta``, ``precision``, ``hbar``.  K is p^2/2."""

    def __init__(self, **kwargs):
        kw = dict(kwargs)
        self.gauge = kw.pop("gauge", "velocity")
        if self.gauge not in ("velocity", "length"):
            raise ValueError("gauge must be 'velocity' or 'length'")
        gamma = kw.get("gamma")
        kw.setdefault("K", lambda _, p: 0.5 * p ** 2)
        kw.setdefault("diff_K", lambda _, p: p)
        super().__init__(**kw)
        if not (hasattr(self, "A") or hasattr(self, "E")):
            raise AttributeError("the laser field was not specified (A(t) or E(t))")
        if self.gauge == "length" and not hasattr(self, "E"):
            raise AttributeError("the length gauge needs E(t)")
        self._A_cache = {}
        self._Aint = (0.0, 0.0)  # (t, A(t)) for the FP64 field integral
        if gamma is not None:
            self.gamma = float(gamma)
            self.w_coeff = np.exp(-self.gamma * 0.5 * self.dt)
            bkw = {k: v for k, v in kwargs.items() if k not in ("gauge", "A", "E", "gamma", "V", "K")}
            t0 = self.t
            V0 = self.V
            if self.gauge == "length":
                E0 = self.field(t0)
                bkw["V"] = lambda _, x: V0(x) + x * E0
                bkw["K"] = lambda _, p: 0.5 * p ** 2
            else:
                A0 = self.vector_potential(t0)
                bkw["V"] = lambda _, x: V0(x)
                bkw["K"] = lambda _, p: 0.5 * (p + A0) ** 2
            g = WignerBlochFFTW1D(**bkw)
            self.gibbs_state = g.get_gibbs_state()
            del g
            self.scaled_gibbs_state = self.gibbs_state * (1 - self.w_coeff)
            if self.isEhrenfest:
                dc = self.scaled_gibbs_state.sum(axis=0)
                self.X_average_gibbs = np.dot(dc / dc.sum(), self.X.reshape(-1))
                dm = self.scaled_gibbs_state.sum(axis=1)
                self.P_average_gibbs = np.dot(dm / dm.sum(), self.P.reshape(-1))
            self._step_kind = FW_STEP_SPLIT
            self._s0 = to_device(self.scaled_gibbs_state, self._rt, self.device)
            self._blend_c = float(self.w_coeff)
        else:
            self.gamma = None

    # -- field ----------------------------------------------------------------
    def vector_potential(self, t):
        """A(t): the user's A, else -int_0^t E (FP64 Gauss-Legendre, advanced incrementally)."""
        if hasattr(self, "A"):
            return float(self.A(t))
        t0, a0 = self._Aint
        if t < t0:
            t0, a0 = 0.0, 0.0
        a = a0 - integrate_field(lambda s: self.E(s), t0, t, pieces=max(1, int(np.ceil((t - t0) / self.dt)) * 2))
        self._Aint = (t, a)
        return a

    def vector_potentials(self, times):
        """A at each of the increasing `times`, as successive vector_potential(t)
        calls return it: the user's A on the whole array, else -int E advanced
        interval by interval (the same composite Gauss-Legendre rule and piece
        counts), with all intervals' quadrature nodes evaluated at once."""
        times = np.asarray(times, dtype=np.float64)
        if hasattr(self, "A"):
            return _on_times(lambda t: self.A(t), times)
        out = np.empty(times.shape)
        out[0] = self.vector_potential(times[0])  # continues (or restarts) the cached integral
        if times.size > 1:
            t0s, t1s = times[:-1], times[1:]
            pieces = np.maximum(1, np.ceil((t1s - t0s) / self.dt).astype(np.int64)) * 2
            inc = np.empty(t0s.shape)
            for pc in np.unique(pieces):
                sel = np.nonzero(pieces == pc)[0]
                inc[sel] = integrate_intervals(lambda u: self.E(u), t0s[sel], t1s[sel], int(pc))
            out[:] = np.cumsum(np.concatenate(([out[0]], -inc)))  # a_k = a_(k-1) - int_k, in order
            self._Aint = (float(times[-1]), float(out[-1]))
        return out

    def fields(self, times):
        """E at each of `times` (one call on the array when E vectorises)."""
        times = np.asarray(times, dtype=np.float64)
        if hasattr(self, "E"):
            return _on_times(lambda t: self.E(t), times)
        return np.array([self.field(t) for t in times])

    def field(self, t):
        if hasattr(self, "E"):
            return float(self.E(t))
        h = 1e-4 * self.dt
        return -(float(self.A(t + h)) - float(self.A(t - h))) / (2 * h)

    # the static parts of the Hamiltonian ----------------------------------------
    def _k_time_dependent(self):
        return False

    def _v_time_dependent(self):
        return False

    def _k_at(self, p, t):
        return np.asarray(0.5 * p ** 2, dtype=np.float64)

    def _tables_static(self):
        return True

    def _propagate_chunk(self, nsteps, t0, tables=None, weights=None, host=True):
        if tables is not None:
            return super()._propagate_chunk(nsteps, t0, tables, weights, host=host)
        times = t0 + self.dt * np.arange(1, nsteps + 1)
        tabV, tabK = self._static_tables()
        if self.gauge == "velocity":
            A = self.vector_potentials(times)
            lam = self.Lambda.reshape(-1)
            g = np.exp(-1j * self.dt * np.outer(A, lam))             # exp(-i dt A(t) lambda)
            self._gK = torch.view_as_real(to_device(g, self._ct, self.device)).contiguous()
            self._gV = None
            self._chunk_field = (A, np.zeros_like(A))
        else:
            E = self.fields(times)
            th = self.Theta.reshape(-1)
            g = np.exp(0.5j * self.dt * np.outer(E, th))             # exp(i dt E(t) theta / 2)
            self._gV = torch.view_as_real(to_device(g, self._ct, self.device)).contiguous()
            self._gK = None
            self._chunk_field = (np.zeros_like(E), E)
        return super()._propagate_chunk(nsteps, t0, tables=(tabV, 0, tabK, 0, False), weights=weights, host=host)

    def _chunk_context(self):
        return getattr(self, "_chunk_field", None)

    def _set_chunk_context(self, ctx):
        self._chunk_field = ctx

    def _chunk_steps(self):
        return 64  # field factors for 64 steps are built while the previous 64 run

    def _weights_at(self, t):
        X, P = self.X.reshape(-1), self.P.reshape(-1)
        E = self.field(t) if self.gauge == "length" else 0.0
        A = self.vector_potential(t) if self.gauge == "velocity" else 0.0
        dv = np.broadcast_to(self.diff_V(self.X), self.X.shape).reshape(-1) + E
        v = np.broadcast_to(self._v_at(self.X, t), self.X.shape).reshape(-1) + E * X
        wx = np.stack([X, dv, v])
        wp = np.stack([P, P + A, 0.5 * (P + A) ** 2])
        return wx, wp

    def _obs_weights(self, times):
        """Static weights [x, V0'(x), V0(x)] and [p, p^2]: the field enters the
        Ehrenfest observables only through the scalars A(t), E(t), applied to
        the recorded sums afterwards (_expand_obs), so no per-step weights."""
        if not self.isEhrenfest:
            return None, None
        if getattr(self, "_obs_static", None) is None:
            X, P = self.X.reshape(-1), self.P.reshape(-1)
            dv = np.broadcast_to(self.diff_V(self.X), self.X.shape).reshape(-1)
            v = np.broadcast_to(self._v_at(self.X, self.t), self.X.shape).reshape(-1)
            wx = to_device(np.stack([X, dv, v]), torch.float64, self.device)
            wp = to_device(np.stack([P, P * P]), torch.float64, self.device)
            self._obs_static = (wx, wp)
        return self._obs_static

    def _expand_obs(self, obs):
        """Sums of the static weights -> the sums _weights_at(t) would give:
        x, V0' + E, V0 + E x and p, p + A, (p + A)^2 / 2 (linear in the sums)."""
        A, E = self._chunk_field
        S, x1, dv, v, p1, p2 = (obs[:, c] for c in (0, 2, 3, 4, 5, 6))
        full = np.empty((obs.shape[0], 8))
        full[:, 0:2] = obs[:, 0:2]
        full[:, 2] = x1
        full[:, 3] = dv + E * S
        full[:, 4] = v + E * x1
        full[:, 5] = p1
        full[:, 6] = p1 + A * S
        full[:, 7] = 0.5 * p2 + A * p1 + 0.5 * A * A * S
        return full

    def _ehrenfest_from_obs(self, obs):
        n = obs.shape[0]
        super()._ehrenfest_from_obs(self._expand_obs(obs))
        if self.gamma is not None:
            for k in range(len(self.X_average) - n, len(self.X_average)):
                self.X_average_RHS[k] += self.gamma * (self.X_average_gibbs - self.X_average[k])
                self.P_average_RHS[k] += self.gamma * (self.P_average_gibbs - self.P_average[k])
