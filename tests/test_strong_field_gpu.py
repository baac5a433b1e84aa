"""Strong-field runs: separable laser field in both gauges, with and without
random-collision dephasing, against the reference fixture and the FP64 oracle."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from cases import CASES, vector_potential  # noqa: E402

from oracle.wigner_oracle import WignerOracle  # noqa: E402

pytestmark = pytest.mark.gpu
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_velocity_gauge_matches_reference_fixture():
    from fastwigner_b200 import StrongFieldWigner

    case = CASES["moyal_velocity_gauge_128x256"]
    g = np.load(ROOT / "tests" / "golden" / "moyal_velocity_gauge_128x256.npz")
    kw = {k: v for k, v in case["kw"].items() if k not in ("K", "diff_K")}
    q = StrongFieldWigner(**kw, gauge="velocity", A=lambda _, t: vector_potential(t))
    q.set_wignerfunction(case["init"])
    W = q.propagate(case["steps"])
    assert rel(W, g["W"]) < 1e-10
    for k in OBS:
        np.testing.assert_allclose(getattr(q, k), g[k], rtol=1e-10, atol=1e-13)


def test_velocity_gauge_from_field_integral():
    """A(t) = -int E: FP64 Gauss-Legendre integral of E(t) = -dA/dt reproduces the closed form."""
    from fastwigner_b200 import StrongFieldWigner

    F, w = 0.04, 0.05698
    E = lambda t: F * (np.cos(w * t) * np.sin(w * t / 16) ** 2  # noqa: E731
                       + np.sin(w * t) * np.sin(w * t / 16) * np.cos(w * t / 16) / 8.0)
    kw = {k: v for k, v in CASES["moyal_velocity_gauge_128x256"]["kw"].items() if k not in ("K", "diff_K", "t")}
    a = StrongFieldWigner(**kw, t=0.0, gauge="velocity", A=lambda _, t: vector_potential(t))
    b = StrongFieldWigner(**kw, t=0.0, gauge="velocity", E=lambda _, t: E(t))
    for q in (a, b):
        q.set_wignerfunction(CASES["moyal_velocity_gauge_128x256"]["init"])
        q.propagate(200)
    assert abs(b.vector_potential(b.t) - vector_potential(b.t)) < 1e-12
    assert rel(b.wignerfunction, a.wignerfunction) < 1e-10


@pytest.mark.parametrize("gamma", [None, 0.05])
def test_length_gauge_soft_core_with_optional_collisions(gamma):
    from fastwigner_b200 import StrongFieldWigner

    E = lambda t: 0.05 * np.sin(np.pi * t / 40.0) ** 2 * np.sin(0.057 * t)  # noqa: E731
    kw = dict(t=2.0, dt=0.05, X_gridDIM=256, X_amplitude=30.0, P_gridDIM=128, P_amplitude=5.0)
    V0 = lambda x: -1.0 / np.sqrt(x * x + 1.0)  # noqa: E731
    dV0 = lambda x: x / (x * x + 1.0) ** 1.5  # noqa: E731
    extra = {} if gamma is None else dict(gamma=gamma, kT=0.5, dbeta=0.01)
    q = StrongFieldWigner(**kw, gauge="length", V=lambda _, x: V0(x), diff_V=lambda _, x: dV0(x),
                          E=lambda _, t: E(t), **extra)
    o = WignerOracle(**kw, V=lambda x, t: V0(x) + x * E(t), K=lambda p: 0.5 * p * p,
                     diff_V=lambda x, t: dV0(x) + E(t), diff_K=lambda p: p)
    if gamma is not None:
        o.setup_collision(gamma, 0.5, 0.01)
    init = lambda _, x, p: np.exp(-(x + 1.0) ** 2 - (p - 0.3) ** 2) + 0 * x * p  # noqa: E731
    q.set_wignerfunction(init)
    o.set_wignerfunction(init(None, o.X, o.P))
    W = q.propagate(30)
    o.propagate(30)
    assert rel(W, o.W) < 1e-10
    for k in OBS:
        np.testing.assert_allclose(getattr(q, k), getattr(o, k), rtol=1e-10, atol=1e-12)
