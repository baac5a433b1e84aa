"""Even grid sizes that are not powers of two (the reference only asserts
evenness: wigner_moyal_fftw_1d.py:55, 62; wigner_moyal_cuda_1d.py:63, 70).
They run the generic mixed-radix passes.  The FFTW-class cases (96 x 192,
100 x 100, 98 x 202 with the absorbing boundary, the Bloch and collision
classes at 160 and 96) are in the golden fixtures recorded from the reference
and run by tests/test_wigner_gpu.py; this file covers the C-string class, a
batch through the per-instance totals path, odd x with a power-of-two p (the
regular row shape is not available) and the x-p mask, against the FP64
oracle at 1e-10 (FP64) and 1e-5 (FP32)."""
import numpy as np
import pytest

from oracle.wigner_oracle import WignerOracle

pytestmark = pytest.mark.gpu


def fw():
    import fastwigner_b200

    return fastwigner_b200


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("P,X", [(96, 160), (256, 100), (120, 128), (18, 30)])
@pytest.mark.parametrize("precision,tol", [("float64", 1e-10), ("float32", 1e-5)])
def test_cuda_class_odd_sizes_match_oracle(P, X, precision, tol):
    kw = dict(t=0.5, dt=0.01, X_gridDIM=X, X_amplitude=9.0, P_gridDIM=P, P_amplitude=8.0)
    q = fw().WignerMoyalCUDA1D(**kw, K="0.5 * P * P", V="0.05 * X * X * X * X - X * X", diff_K="P",
                               diff_V="0.2 * X * X * X - 2.0 * X",
                               abs_boundary_x_p="pow(abs(sin(0.5 * M_PI * (X + X_amplitude) / X_amplitude)), dt * 0.5)",
                               precision=precision)
    q.set_wignerfunction("exp(-(X - 1.0) * (X - 1.0) - 2.0 * (P + 0.5) * (P + 0.5))")
    o = WignerOracle(**kw, convention="cuda", V=lambda x: 0.05 * x ** 4 - x * x, K=lambda p: 0.5 * p * p,
                     diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p,
                     abs_boundary_x_p=lambda X_, P_: np.abs(np.sin(0.5 * np.pi * (X_ + 9.0) / 9.0)) ** (0.01 * 0.5)
                     + 0 * P_)
    o.set_wignerfunction(np.exp(-(o.X - 1.0) ** 2 - 2.0 * (o.P + 0.5) ** 2))
    W = q.propagate(12).get()
    o.propagate(12)
    assert rel(W, o.W) < tol
    for k in ("X_average", "P_average", "hamiltonian_average"):
        np.testing.assert_allclose(getattr(q, k), getattr(o, k), rtol=10 * tol, atol=10 * tol)


def test_batch_of_odd_grids_through_the_totals_path():
    """A 6-instance FP64 batch on a 150 x 210 grid (per-instance totals kernel,
    fused observables through the generic column pass's real-space sums)."""
    from fastwigner_b200.batch import WignerMoyalBatch

    B, P, X, steps = 6, 150, 210, 10
    V = lambda x: 0.05 * x ** 4 - x ** 2  # noqa: E731
    K = lambda p: 0.5 * p ** 2  # noqa: E731
    b = WignerMoyalBatch(batch=B, X_gridDIM=X, X_amplitude=10.0, P_gridDIM=P, P_amplitude=10.0, dt=0.005, V=V, K=K,
                         diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p, precision="float64")
    rng = np.random.default_rng(4)
    W0 = np.stack([np.exp(-(b.X - rng.uniform(-2, 2)) ** 2 - (b.P - rng.uniform(-1, 1)) ** 2) for _ in range(B)])
    b.set_wignerfunctions(W0)
    obs = b.propagate(steps).cpu().numpy()
    for i in range(B):
        o = WignerOracle(X_gridDIM=X, X_amplitude=10.0, P_gridDIM=P, P_amplitude=10.0, dt=0.005, V=V, K=K,
                         diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p)
        o.set_wignerfunction(W0[i])
        o.propagate(steps)
        assert rel(b.W[i].cpu().numpy(), o.W) < 1e-10
        np.testing.assert_allclose(obs[:, i, 2] / obs[:, i, 0], o.X_average, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose((obs[:, i, 4] + obs[:, i, 7]) / obs[:, i, 0], o.hamiltonian_average, rtol=1e-10)
