"""GPU parity of the C-string Wigner drop-ins (WignerMoyalCUDA1D,
WignerBlochCUDA1D) against the FP64 oracle in the CUDA-class convention and
the reference fixtures.  FP64 tolerance 1e-10 relative."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from cases import CASES, coherent  # noqa: E402

from oracle.wigner_oracle import WignerOracle, exact_harmonic_gibbs  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = ROOT / "tests" / "golden"
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")
TOL = 1e-10


def fw():
    import fastwigner_b200

    return fastwigner_b200


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


GRID = dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0)


def test_static_hamiltonian_matches_reference_fixture():
    """CUDA-class algorithm == FFTW algorithm for a static Hamiltonian; pin on the fixture."""
    g = np.load(GOLD / "moyal_harmonic_128.npz")
    q = fw().WignerMoyalCUDA1D(**GRID, K="0.5 * P * P", V="0.5 * X * X", diff_K="P", diff_V="X")
    q.set_wignerfunction(CASES["moyal_harmonic_128"]["init"])
    W = q.propagate(20).get()
    assert rel_l2(W, g["W"]) < TOL
    for k in OBS:
        np.testing.assert_allclose(getattr(q, k), g[k], rtol=TOL, atol=1e-13)


def test_time_dependent_field_boundaries_and_c_string_init():
    """Length-gauge field V = V0(x) + x E(t) (t + dt/2 convention), all three
    absorbing-boundary strings, a C-string initial state; vs the oracle."""
    kw = dict(t=3.0, dt=0.02, X_gridDIM=256, X_amplitude=12.0, P_gridDIM=128, P_amplitude=6.0, F=0.3, omega=0.7)
    E = lambda t: -0.3 * np.sin(0.7 * t) * np.sin(0.7 * t / 16.0) ** 2  # noqa: E731
    q = fw().WignerMoyalCUDA1D(
        **kw, functions="__device__ double E(double t){ return -F * sin(omega * t) * pow(sin(omega * t / 16.), 2); }",
        K="0.5 * P * P", V="-1. / sqrt(X * X + 1.37) + X * E(t)",
        diff_K="P", diff_V="X / pow(X * X + 1.37, 1.5) + E(t)",
        abs_boundary_x_theta="exp(-1e-4 * Theta * Theta)",
        abs_boundary_lambda_p="exp(-1e-4 * Lambda * Lambda)",
        abs_boundary_x_p="pow(abs(sin(0.5 * M_PI * (X + X_amplitude) / X_amplitude)), dt * 0.5)")
    q.set_wignerfunction("exp(-(X - 1.0) * (X - 1.0) - 2.0 * P * P)")
    o = WignerOracle(**{k: v for k, v in kw.items() if k not in ("F", "omega")}, convention="cuda",
                     V=lambda x, t: -1.0 / np.sqrt(x * x + 1.37) + x * E(t), K=lambda p: 0.5 * p * p,
                     diff_V=lambda x, t: x / (x * x + 1.37) ** 1.5 + E(t), diff_K=lambda p: p,
                     abs_boundary_x_theta=lambda X, Th: np.exp(-1e-4 * Th * Th) + 0 * X,
                     abs_boundary_lambda_p=lambda L, P: np.exp(-1e-4 * L * L) + 0 * P,
                     abs_boundary_x_p=lambda X, P: np.abs(np.sin(0.5 * np.pi * (X + 12.0) / 12.0)) ** (0.02 * 0.5) + 0 * P)
    o.set_wignerfunction(np.exp(-(o.X - 1.0) ** 2 - 2.0 * o.P ** 2))
    assert rel_l2(q.wignerfunction.get(), o.W) < 1e-13
    W = q.propagate(15).get()
    o.propagate(15)
    assert rel_l2(W, o.W) < TOL
    np.testing.assert_allclose(q.X_average, o.X_average, rtol=TOL, atol=1e-13)
    np.testing.assert_allclose(q.P_average_RHS, o.P_average_RHS, rtol=TOL, atol=1e-13)
    np.testing.assert_allclose(q.hamiltonian_average, o.hamiltonian_average, rtol=TOL, atol=1e-13)


def test_get_average_purity_and_single_step_factor():
    q = fw().WignerMoyalCUDA1D(**GRID, K="0.5 * P * P", V="0.5 * X * X")
    q.set_wignerfunction(coherent(1.0, 0.5))
    q.propagate(5)
    W = q.wignerfunction.get()
    X = q.dX * (np.arange(128) - 64)[None, :]
    P = q.dP * (np.arange(128) - 64)[:, None]
    assert abs(q.get_average("X * P") - np.sum(W * X * P) * q.dXdP) < 1e-13
    assert abs(q.get_purity() - 2 * np.pi * np.sum(W ** 2) * q.dXdP) < 1e-13
    assert abs(q.get_sigma_x_sigma_p() - 0.5) < 1e-6
    # the reference's single step is unnormalised by the three cuFFT inverses (P * X * P)
    o = WignerOracle(**GRID, convention="cuda", V=lambda x: 0.5 * x * x, K=lambda p: 0.5 * p * p)
    o.set_wignerfunction(W)
    o.t = q.t = q.t + q.dt
    o.single_step()
    W1 = q.single_step_propagation().get()
    assert rel_l2(W1, o.W * 128 * 128 * 128) < 1e-12


def test_bloch_cuda_gibbs_pinned_on_fftw_fixture():
    """BlochCUDA(kT/2, 2 dbeta) runs the reference FFTW class's exponents at (kT, dbeta)."""
    g = np.load(GOLD / "bloch_fftw_harmonic_128.npz")
    b = fw().WignerBlochCUDA1D(**GRID, K="0.5 * P * P", V="0.5 * X * X", t_initial=0.0)
    W = b.get_gibbs_state(kT=0.25, dbeta=0.02).get()
    assert rel_l2(W, g["W"]) < TOL


def test_bloch_cuda_exact_gibbs_and_ground_state():
    b = fw().WignerBlochCUDA1D(**{**GRID, "X_gridDIM": 256, "P_gridDIM": 256}, K="0.5 * P * P", V="0.5 * X * X",
                               kT=0.5, dbeta=0.005, t_initial=0.0)
    W = b.get_gibbs_state().get()
    X = b.dX * (np.arange(256) - 128)[None, :]
    P = b.dP * (np.arange(256) - 128)[:, None]
    assert np.abs(exact_harmonic_gibbs(1.0, 0.5, X, P) - W).max() * b.dXdP < 1e-6
    Wg = b.get_ground_state(dbeta=0.05, abs_tol_purity=1e-9).get()
    ground = np.exp(-X ** 2 - P ** 2) / np.pi
    assert np.abs(ground - Wg).max() * b.dXdP < 1e-6
    assert abs(b.get_purity() - 1) < 1e-8
