"""Host-side pieces of the strong-field driver (no GPU): the vectorised FP64
field integral and the expansion of static-weight observable sums."""
import math
import types

import numpy as np
import pytest

from fastwigner_b200.strong_field import StrongFieldWigner, integrate_field, integrate_intervals

E0, W0, TP = 0.07, 0.057, 8 * 2 * math.pi / 0.057


def E_vec(t):
    return E0 * np.sin(np.pi * t / TP) ** 2 * np.sin(W0 * t)


def E_1d(t):  # takes the 8 nodes of one interval but no larger arrays: the per-interval fallback
    t = np.asarray(t)
    if t.ndim != 1:
        raise ValueError("one-dimensional arrays only")
    return np.array([E0 * math.sin(math.pi * u / TP) ** 2 * math.sin(W0 * u) for u in t])


@pytest.mark.parametrize("pieces", [1, 2, 4])
@pytest.mark.parametrize("E", [E_vec, E_1d])
def test_intervals_match_the_scalar_rule(pieces, E):
    rng = np.random.default_rng(0)
    t0 = np.sort(rng.uniform(0, 800, 50))
    t1 = t0 + rng.uniform(0.01, 0.2, 50)
    ref = np.array([integrate_field(E, a, b, pieces) for a, b in zip(t0, t1)])
    got = integrate_intervals(E, t0, t1, pieces)
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=1e-18)


def _namespace(dt):
    ns = types.SimpleNamespace(E=E_vec, dt=dt, _Aint=(0.0, 0.0))
    ns.vector_potential = lambda t: StrongFieldWigner.vector_potential(ns, t)
    return ns


def test_vector_potentials_follow_successive_calls():
    dt = 0.05
    times = 3.0 + dt * np.arange(1, 401)
    a = _namespace(dt)
    ref = np.array([a.vector_potential(t) for t in times])
    b = _namespace(dt)
    got = StrongFieldWigner.vector_potentials(b, times)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)
    assert b._Aint[0] == times[-1] and abs(b._Aint[1] - ref[-1]) < 1e-15
    # the cache continues: the next chunk starts where this one ended
    more = times[-1] + dt * np.arange(1, 11)
    np.testing.assert_allclose(StrongFieldWigner.vector_potentials(b, more),
                               np.array([a.vector_potential(t) for t in more]), rtol=1e-12, atol=1e-15)


def test_static_weight_sums_expand_to_the_field_weights():
    rng = np.random.default_rng(1)
    P, X, n = 16, 32, 5
    x, p = np.linspace(-5, 5, X), np.linspace(-3, 3, P)
    V0, dV0 = -1 / np.sqrt(x * x + 1), x / (x * x + 1) ** 1.5
    Ws = rng.uniform(0, 1, (n, P, X))
    A, E = rng.normal(size=n), rng.normal(size=n)
    obs = np.empty((n, 7))
    full = np.empty((n, 8))
    for k in range(n):
        W = Ws[k]
        mx, mp = W.sum(axis=0), W.sum(axis=1)
        obs[k] = [W.sum(), (W * W).sum(), mx @ x, mx @ dV0, mx @ V0, mp @ p, mp @ (p * p)]
        full[k] = [W.sum(), (W * W).sum(), mx @ x, mx @ (dV0 + E[k]), mx @ (V0 + E[k] * x),
                   mp @ p, mp @ (p + A[k]), mp @ (0.5 * (p + A[k]) ** 2)]
    ns = types.SimpleNamespace(_chunk_field=(A, E))
    np.testing.assert_allclose(StrongFieldWigner._expand_obs(ns, obs), full, rtol=1e-12, atol=1e-12)
