"""Pin the numpy oracle against fixtures recorded from the reference's own classes."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from cases import CASES, CONFIG1  # noqa: E402

from oracle.wigner_oracle import WignerOracle, exact_harmonic_gibbs  # noqa: E402

GOLD = ROOT / "tests" / "golden"
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")


def oracle_for(case):
    kw = {k: v for k, v in case["kw"].items()}
    gamma, kT, dbeta = kw.pop("gamma", None), kw.pop("kT", None), kw.pop("dbeta", 0.01)
    wrap = {}
    for name in ("V", "K", "diff_V", "diff_K"):
        if name in kw:
            f = kw.pop(name)
            wrap[name] = (lambda f: (lambda *a: f(None, *a)))(f)
    o = WignerOracle(**kw, **wrap)
    if case["cls"] == "WignerBlochFFTW1D":
        o.setup_bloch_fftw(kT, dbeta)
    if gamma is not None:
        o.setup_collision(gamma, kT, dbeta)
    return o


def run_oracle(case):
    o = oracle_for(case)
    if case["cls"] == "WignerBlochFFTW1D":
        o.get_gibbs_state_fftw()
        return o
    o.set_wignerfunction(case["init"](o, o.X, o.P))
    o.propagate(case["steps"])
    return o


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    g = np.load(GOLD / f"{name}.npz")
    o = run_oracle(CASES[name])
    rel = np.linalg.norm(o.W - g["W"]) / np.linalg.norm(g["W"])
    assert rel < 1e-12, rel
    for k in OBS:
        if k in g:
            np.testing.assert_allclose(getattr(o, k), g[k], rtol=1e-10, atol=1e-12)


def test_oracle_config1_full_size():
    g = np.load(GOLD / "config1_moyal_256.npz")
    o = run_oracle(CONFIG1)
    for k in OBS:
        np.testing.assert_allclose(getattr(o, k), g[k], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(np.sum(o.W ** 2), g["W_sum_sq"], rtol=1e-10)
    np.testing.assert_allclose(o.W.sum(axis=1), g["W_row_sums"], rtol=1e-9, atol=1e-14)


def test_fftw_bloch_factor_two_quirk():
    """The FFTW Bloch exponents are twice the CUDA class's: the fixture equals the
    exact Gibbs state at kT/2 (wigner_bloch_fftw_1d.py:75,96 vs wigner_bloch_cuda_1d.py:299,338)."""
    g = np.load(GOLD / "bloch_fftw_harmonic_128.npz")
    o = oracle_for(CASES["bloch_fftw_harmonic_128"])
    kT = CASES["bloch_fftw_harmonic_128"]["kw"]["kT"]
    err_half = np.abs(exact_harmonic_gibbs(1.0, kT / 2, o.X, o.P) - g["W"]).max() * o.dXdP
    err_full = np.abs(exact_harmonic_gibbs(1.0, kT, o.X, o.P) - g["W"]).max() * o.dXdP
    assert err_half < 1e-7 and err_full > 1e-5


def test_cuda_bloch_restatement_equals_fftw_at_half_temperature():
    """Pins the CUDA-class Bloch restatement: BlochCUDA(kT/2, 2*dbeta) runs the same
    exponents as the reference FFTW class at (kT, dbeta)."""
    case = CASES["bloch_fftw_harmonic_128"]
    g = np.load(GOLD / "bloch_fftw_harmonic_128.npz")
    kw = {k: v for k, v in case["kw"].items() if k not in ("kT", "dbeta")}
    V, K = kw.pop("V"), kw.pop("K")
    o = WignerOracle(**kw, V=lambda x: V(None, x), K=lambda p: K(None, p), convention="fftw")
    o.setup_bloch_cuda(0.0)
    o.get_gibbs_state_cuda(case["kw"]["kT"] / 2, 2 * case["kw"]["dbeta"])
    rel = np.linalg.norm(o.W - g["W"]) / np.linalg.norm(g["W"])
    assert rel < 1e-11, rel


def test_cuda_convention_equals_fftw_for_static_hamiltonian():
    """For a time-independent Hamiltonian the CUDA-class restatement (positive
    Nyquist, t + dt/2, index-formula grids) is the FFTW algorithm: pin it on the golden."""
    case = CASES["moyal_harmonic_128"]
    g = np.load(GOLD / "moyal_harmonic_128.npz")
    kw = dict(case["kw"])
    wrap = {n: (lambda f: (lambda *a: f(None, *a)))(kw.pop(n)) for n in ("V", "K", "diff_V", "diff_K")}
    o = WignerOracle(**kw, **wrap, convention="cuda")
    o.set_wignerfunction(case["init"](o, o.X, o.P))
    o.propagate(case["steps"])
    rel = np.linalg.norm(o.W - g["W"]) / np.linalg.norm(g["W"])
    assert rel < 1e-12, rel
