"""Known-answer checks that pin the density-matrix oracle (the reference's
RhoVNeumannCUDA1D / RhoBlochCUDA1D need PyCUDA and a GPU, so there is no
reference run to record fixtures from; these are the checks its demos make)."""
import numpy as np

from oracle.rho_oracle import RhoOracle
from oracle.wigner_oracle import exact_harmonic_gibbs


def test_bloch_gibbs_wigner_matches_exact_harmonic():
    """rho_bloch_cuda_1d.py:404-424: W of the Bloch Gibbs state vs the exact
    harmonic-oscillator Gibbs Wigner function (inf-norm * wigner_dxdp)."""
    kT = 0.5
    o = RhoOracle(X_gridDIM=256, X_amplitude=12.0, dt=0.01, V=lambda x: 0.5 * x * x, K=lambda p: 0.5 * p * p)
    o.setup_bloch(0.0)
    o.get_gibbs_state(kT, 0.005)
    W = o.get_wignerfunction().real
    exact = exact_harmonic_gibbs(1.0, kT, o.X_wigner, o.P_wigner)
    assert np.abs(W - exact).max() * o.wigner_dxdp < 1e-4


def test_von_neumann_coherent_state_follows_classical_orbit():
    """Harmonic oscillator: <x>(t) = x0 cos t + p0 sin t for a coherent state."""
    x0, p0 = 1.0, 0.5
    o = RhoOracle(X_gridDIM=256, X_amplitude=12.0, dt=0.01, V=lambda x: 0.5 * x * x, K=lambda p: 0.5 * p * p,
                  diff_V=lambda x, t: x, diff_K=lambda p, t: p)
    X = o.X
    psi = np.exp(-0.5 * (X - x0) ** 2 + 1j * p0 * X)
    o.set_rho(np.outer(np.conj(psi), psi))
    o.propagate(200)
    t = 0.01 * np.arange(1, 201)
    np.testing.assert_allclose(o.X_average, x0 * np.cos(t) + p0 * np.sin(t), atol=1e-4)
    h = np.array(o.hamiltonian_average)
    assert (1 - h.min() / h.max()) < 5e-5  # split-operator energy error is O(dt^2), not zero
