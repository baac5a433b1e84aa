"""Pin the CUDA-convention oracles against fixtures recorded from the
reference's own CUDA classes (tests/golden/gen_golden_cuda.py: the unmodified
RhoVNeumannCUDA1D, RhoBlochCUDA1D, WignerMoyalCUDA1D and WignerBlochCUDA1D,
their kernel strings compiled for the host, cuFFT's unnormalised conventions
on pocketfft).  Tolerance 1e-12 relative (FP64 restatement vs FP64 reference
run; the reference prints its constants with 16 significant digits)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))

from oracle.rho_oracle import RhoOracle  # noqa: E402
from oracle.wigner_oracle import WignerOracle  # noqa: E402

GOLD = ROOT / "tests" / "golden"
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")
TOL = 1e-12


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def load(name):
    return np.load(GOLD / f"cuda_{name}.npz")


def _E(F, omega):
    return lambda t: -F * np.sin(omega * t) * np.sin(omega * t / 16.0) ** 2


def _rho_dw():
    return dict(V=lambda x: 0.05 * x ** 4 - x ** 2, K=lambda p: 0.5 * p * p,
                diff_V=lambda x, t: 0.2 * x ** 3 - 2 * x, diff_K=lambda p, t: p)


def _check_rho_run(o, g, steps, Ip, H):
    o.set_rho(g["rho0"])
    wi = g["wigner_initial"]
    wt = []
    for _ in range(steps):
        o.propagate(1)
        wt.append(o.get_wigner_time(o.get_wignerfunction(), wi, o.t, Ip, H))
    assert abs(o.t - float(g["t"])) < 1e-12
    assert rel(o.rho, g["rho"]) < TOL
    for k in OBS:
        np.testing.assert_allclose(getattr(o, k), g[k], rtol=TOL, atol=1e-13)
    np.testing.assert_allclose(wt, g["wigner_time"], rtol=1e-10, atol=1e-13)
    assert abs(o.get_purity() - float(g["purity"])) < 1e-13
    assert rel(o.get_wignerfunction(), g["W"]) < TOL


def test_rho_von_neumann_double_well():
    g = load("rho_vn_dw_128")
    o = RhoOracle(t=0.0, dt=0.005, X_gridDIM=128, X_amplitude=10.0, **_rho_dw())
    H = lambda X, P, t: 0.5 * P * P + 0.05 * X ** 4 - X * X  # noqa: E731
    _check_rho_run(o, g, 25, 0.4, H)


def test_rho_von_neumann_field_and_absorbers():
    g = load("rho_vn_field_abs_128")
    E = _E(0.2, 0.3)
    o = RhoOracle(t=5.0, dt=0.02, X_gridDIM=128, X_amplitude=10.0,
                  V=lambda x, t: -1.0 / np.sqrt(x * x + 1.37) + x * E(t), K=lambda p: 0.5 * p * p,
                  diff_V=lambda x, t: x / (x * x + 1.37) ** 1.5 + E(t), diff_K=lambda p, t: p,
                  abs_boundary_x=lambda X, Xp: np.abs(np.sin(0.5 * np.pi * (X + 10) / 10)
                                                      * np.sin(0.5 * np.pi * (Xp + 10) / 10)) ** (0.02 * 0.05),
                  abs_boundary_p=lambda P, Pp: np.exp(-1e-3 * 0.02 * (P * P + Pp * Pp)))
    H = lambda X, P, t: 0.5 * P * P - 1.0 / np.sqrt(X * X + 1.37) + X * E(t)  # noqa: E731
    _check_rho_run(o, g, 15, 0.5, H)


def test_rho_bloch_gibbs_with_the_reference_k_min():
    g = load("rho_bloch_gibbs_dw_128")
    o = RhoOracle(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, V=lambda x: 0.05 * x ** 4 - x ** 2,
                  K=lambda p: 0.5 * p * p)
    o.setup_bloch(0.0)
    o.get_gibbs_state(0.5, 0.01)
    assert rel(o.rho, g["rho"]) < TOL
    assert rel(o.get_wignerfunction(), g["W"]) < TOL
    assert abs(o.get_purity() - float(g["purity"])) < 1e-13


def test_rho_bloch_ground_state_rollback():
    g = load("rho_bloch_ground_harmonic_128")
    o = RhoOracle(t=0.0, dt=0.05, X_gridDIM=128, X_amplitude=8.0, V=lambda x: 0.5 * x * x,
                  K=lambda p: 0.5 * p * p)
    o.setup_bloch(0.0)
    o.get_ground_state(0.1, 1e-9)
    assert rel(o.rho, g["rho"]) < 1e-10
    assert abs(o.get_purity() - float(g["purity"])) < 1e-12


def test_wigner_cuda_field_and_three_absorbers():
    g = load("wigner_cuda_field_abs_256x128")
    E = _E(0.3, 0.7)
    o = WignerOracle(t=3.0, dt=0.02, X_gridDIM=256, X_amplitude=12.0, P_gridDIM=128, P_amplitude=6.0,
                     convention="cuda", V=lambda x, t: -1.0 / np.sqrt(x * x + 1.37) + x * E(t),
                     K=lambda p: 0.5 * p * p, diff_V=lambda x, t: x / (x * x + 1.37) ** 1.5 + E(t),
                     diff_K=lambda p: p,
                     abs_boundary_x_theta=lambda X, Th: np.exp(-1e-4 * Th * Th) + 0 * X,
                     abs_boundary_lambda_p=lambda L, P: np.exp(-1e-4 * L * L) + 0 * P,
                     abs_boundary_x_p=lambda X, P: np.abs(np.sin(0.5 * np.pi * (X + 12.0) / 12.0)) ** (0.02 * 0.5)
                     + 0 * P)
    o.set_wignerfunction(g["W0"])
    o.propagate(15)
    assert rel(o.W, g["W"]) < TOL
    for k in OBS:
        np.testing.assert_allclose(getattr(o, k), g[k], rtol=TOL, atol=1e-13)


def test_wigner_bloch_cuda_gibbs():
    g = load("wigner_bloch_cuda_dw_128")
    o = WignerOracle(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0,
                     convention="cuda", V=lambda x: 0.05 * x ** 4 - x ** 2, K=lambda p: 0.5 * p * p)
    o.setup_bloch_cuda(0.0)
    o.get_gibbs_state_cuda(0.5, 0.01)
    assert rel(o.W, g["W_gibbs"]) < TOL


def test_wigner_bloch_cuda_ground_state_rollback():
    g = load("wigner_bloch_cuda_ground_harmonic_128")
    o = WignerOracle(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0,
                     convention="cuda", V=lambda x: 0.5 * x * x, K=lambda p: 0.5 * p * p)
    o.setup_bloch_cuda(0.0)
    o.get_ground_state_cuda(0.05, 1e-9)
    assert rel(o.W, g["W_ground"]) < 1e-10
    assert abs(o.get_purity() - float(g["purity_ground"])) < 1e-12


@pytest.mark.parametrize("name", ["rho_vn_dw_128", "rho_vn_field_abs_128", "rho_bloch_gibbs_dw_128",
                                  "rho_bloch_ground_harmonic_128", "wigner_cuda_field_abs_256x128",
                                  "wigner_bloch_cuda_dw_128", "wigner_bloch_cuda_ground_harmonic_128"])
def test_fixture_present_and_finite(name):
    g = load(name)
    for k in g.files:
        assert np.all(np.isfinite(g[k])), k
