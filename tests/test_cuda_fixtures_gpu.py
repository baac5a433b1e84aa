"""GPU parity of the C-string drop-ins (RhoVNeumannCUDA1D, RhoBlochCUDA1D,
WignerMoyalCUDA1D, WignerBlochCUDA1D) against fixtures recorded from the
reference's own CUDA classes (tests/golden/gen_golden_cuda.py), with the same
constructor keywords and C strings.  FP64, tolerance 1e-10 relative."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from cases_cuda import CUDA_CASES  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = ROOT / "tests" / "golden"
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")
TOL = 1e-10


def fw():
    import fastwigner_b200

    return fastwigner_b200


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _get(x):
    return np.asarray(x.get() if hasattr(x, "get") else x)


@pytest.mark.parametrize("name", ["rho_vn_dw_128", "rho_vn_field_abs_128"])
def test_von_neumann_matches_reference_cuda_fixture(name):
    case = CUDA_CASES[name]
    g = np.load(GOLD / f"cuda_{name}.npz")
    q = getattr(fw(), case["cls"])(**dict(case["kw"]))
    q.set_rho(case["init"])
    assert rel(_get(q.rho), g["rho0"]) < 1e-13
    q.wigner_initial = g["wigner_initial"]
    q.propagate(case["steps"])
    assert abs(q.t - float(g["t"])) < 1e-12
    assert rel(_get(q.rho), g["rho"]) < TOL
    for k in OBS:
        np.testing.assert_allclose(getattr(q, k), g[k], rtol=TOL, atol=1e-12, err_msg=k)
    np.testing.assert_allclose(q.wigner_time, g["wigner_time"], rtol=1e-9, atol=1e-12)
    assert abs(q.get_purity() - float(g["purity"])) < 1e-11
    assert rel(_get(q.get_wignerfunction()), g["W"]) < TOL
    assert abs(q.get_sigma_x_sigma_p() - float(g["sigma_x_sigma_p"])) < 1e-9


def test_rho_bloch_gibbs_matches_reference_cuda_fixture():
    case = CUDA_CASES["rho_bloch_gibbs_dw_128"]
    g = np.load(GOLD / "cuda_rho_bloch_gibbs_dw_128.npz")
    q = fw().RhoBlochCUDA1D(**dict(case["kw"]))
    q.get_gibbs_state(**case["gibbs"])
    assert rel(_get(q.rho), g["rho"]) < TOL
    assert rel(_get(q.get_wignerfunction()), g["W"]) < TOL
    assert abs(q.get_purity() - float(g["purity"])) < 1e-11


def test_rho_bloch_ground_state_matches_reference_cuda_fixture():
    case = CUDA_CASES["rho_bloch_ground_harmonic_128"]
    g = np.load(GOLD / "cuda_rho_bloch_ground_harmonic_128.npz")
    q = fw().RhoBlochCUDA1D(**dict(case["kw"]))
    q.get_ground_state(**case["ground"])
    assert rel(_get(q.rho), g["rho"]) < 1e-9
    assert abs(q.get_purity() - float(g["purity"])) < 1e-10


def test_wigner_cuda_matches_reference_cuda_fixture():
    case = CUDA_CASES["wigner_cuda_field_abs_256x128"]
    g = np.load(GOLD / "cuda_wigner_cuda_field_abs_256x128.npz")
    q = fw().WignerMoyalCUDA1D(**dict(case["kw"]))
    q.set_wignerfunction(case["init"])
    assert rel(_get(q.wignerfunction), g["W0"]) < 1e-13
    q.propagate(case["steps"])
    assert rel(_get(q.wignerfunction), g["W"]) < TOL
    for k in OBS:
        np.testing.assert_allclose(getattr(q, k), g[k], rtol=TOL, atol=1e-12, err_msg=k)
    assert abs(q.get_purity() - float(g["purity"])) < 1e-11


def test_wigner_bloch_cuda_matches_reference_cuda_fixtures():
    case = CUDA_CASES["wigner_bloch_cuda_dw_128"]
    g = np.load(GOLD / "cuda_wigner_bloch_cuda_dw_128.npz")
    q = fw().WignerBlochCUDA1D(**dict(case["kw"]))
    assert rel(_get(q.get_gibbs_state(**case["gibbs"])), g["W_gibbs"]) < TOL
    case = CUDA_CASES["wigner_bloch_cuda_ground_harmonic_128"]
    g = np.load(GOLD / "cuda_wigner_bloch_cuda_ground_harmonic_128.npz")
    q = fw().WignerBlochCUDA1D(**dict(case["kw"]))
    assert rel(_get(q.get_ground_state(**case["ground"])), g["W_ground"]) < 1e-9
    assert abs(q.get_purity() - float(g["purity_ground"])) < 1e-10
