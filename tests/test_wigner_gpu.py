"""GPU parity of the Wigner-function drop-ins against the reference fixtures
and the FP64 oracle.

Tolerances (tests/parity_tables.py): FP64 runs 1e-10 relative (L2 of W and
every observable); FP32 runs (complex64 spectra, FP64-built phases) 1e-5
relative L2 of W and FP32_OBS_TOL per observable."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from cases import CASES, CONFIG1  # noqa: E402

from oracle.wigner_oracle import WignerOracle, exact_harmonic_gibbs  # noqa: E402

sys.path.insert(0, str(ROOT / "tests"))
from parity_tables import FP32_OBS_TOL, FP32_TOL, FP64_TOL  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = ROOT / "tests" / "golden"
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")


def fw():
    import fastwigner_b200

    return fastwigner_b200


def build(case, precision):
    cls = getattr(fw(), case["cls"])
    return cls(**case["kw"], precision=precision)


def run(case, precision):
    obj = build(case, precision)
    if case["cls"] == "WignerBlochFFTW1D":
        return obj, obj.get_gibbs_state()
    obj.set_wignerfunction(case["init"])
    return obj, obj.propagate(case["steps"])


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_reference_fixture(name):
    g = np.load(GOLD / f"{name}.npz")
    obj, W = run(CASES[name], "float64")
    assert rel_l2(W, g["W"]) < FP64_TOL
    for k in OBS:
        if k in g:
            np.testing.assert_allclose(getattr(obj, k), g[k], rtol=FP64_TOL, atol=1e-13)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32_matches_reference_fixture(name):
    g = np.load(GOLD / f"{name}.npz")
    obj, W = run(CASES[name], "float32")
    assert rel_l2(W, g["W"]) < FP32_TOL
    for k in OBS:
        if k in g:
            rtol, atol = FP32_OBS_TOL[k]
            np.testing.assert_allclose(getattr(obj, k), g[k], rtol=rtol, atol=atol)


def test_config1_fp64_1000_steps():
    g = np.load(GOLD / "config1_moyal_256.npz")
    obj, W = run(CONFIG1, "float64")
    for k in OBS:
        np.testing.assert_allclose(getattr(obj, k), g[k], rtol=FP64_TOL, atol=1e-13)
    np.testing.assert_allclose(np.sum(W ** 2), g["W_sum_sq"], rtol=FP64_TOL)
    cs = g["W_col_sums"]
    np.testing.assert_allclose(W.sum(axis=0), cs, rtol=0, atol=FP64_TOL * np.abs(cs).max())


def test_propagate_in_chunks_equals_one_call():
    case = CASES["moyal_harmonic_128"]
    a, Wa = run(case, "float64")
    b = build(case, "float64")
    b.set_wignerfunction(case["init"])
    for _ in range(case["steps"] // 5):
        Wb = b.propagate(5)
    assert rel_l2(Wb, Wa) < 1e-13
    np.testing.assert_allclose(b.X_average, a.X_average, rtol=1e-13)


def test_single_step_is_unnormalised_step():
    case = CASES["moyal_dw_alpha_128x256"]
    obj = build(case, "float64")
    obj.set_wignerfunction(case["init"])
    o = WignerOracle(**{k: v for k, v in case["kw"].items() if k not in ("V", "K", "diff_V", "diff_K")},
                     V=lambda x: case["kw"]["V"](None, x), K=lambda p: case["kw"]["K"](None, p))
    o.set_wignerfunction(obj.wignerfunction)
    o.t += o.dt  # the reference evaluates the exponents at the (incremented) current time
    obj.t += obj.dt
    o.single_step()
    W = obj.single_step_propagation()
    assert rel_l2(W, o.W) < 1e-12


def test_purity_average_sigma():
    case = CASES["moyal_harmonic_128"]
    obj, W = run(case, "float64")
    o = WignerOracle(**{k: v for k, v in case["kw"].items() if k not in ("V", "K", "diff_V", "diff_K")},
                     V=lambda x: 0.5 * x ** 2, K=lambda p: 0.5 * p ** 2)
    o.set_wignerfunction(W)
    assert abs(obj.get_purity() - o.get_purity()) < 1e-12
    assert abs(obj.get_average(lambda self, x, p: x * p) - o.get_average(lambda x, p: x * p)) < 1e-12
    # coherent state of the harmonic oscillator: sigma_x sigma_p = 1/2
    assert abs(obj.get_sigma_x_sigma_p() - 0.5) < 1e-6


def test_bloch_fftw_matches_exact_gibbs_at_half_temperature():
    case = CASES["bloch_fftw_harmonic_128"]
    obj, W = run(case, "float64")
    kT = case["kw"]["kT"]
    err = np.abs(exact_harmonic_gibbs(1.0, kT / 2, obj.X, obj.P) - W).max() * obj.dXdP
    assert err < 1e-7


def test_errors_like_reference():
    kw = dict(CASES["moyal_harmonic_128"]["kw"])
    with pytest.raises(AssertionError):
        fw().WignerMoyalFTTW1D(**{**kw, "X_gridDIM": 127})
    kw.pop("dt")
    with pytest.raises(AttributeError):
        fw().WignerMoyalFTTW1D(**kw)
    obj = build(CASES["moyal_harmonic_128"], "float64")
    with pytest.raises(AssertionError):
        obj.set_wignerfunction(np.zeros((4, 4)))
    with pytest.raises(NotImplementedError):
        obj.set_wignerfunction("not a function")


@pytest.mark.parametrize("P", [256, 512, 1024])
def test_fp32_larger_grids_match_oracle(P):
    """FP32 parity with the FP64 oracle on the grid sizes of the benchmark workloads."""
    kw = dict(t=0.0, dt=0.005, X_gridDIM=256, X_amplitude=10.0, P_gridDIM=P, P_amplitude=10.0)
    V = lambda x: 0.05 * x ** 4 - x ** 2  # noqa: E731
    init = lambda x, p: np.exp(-(x + 1.3) ** 2 / 0.25 - 0.25 * (p - 0.4) ** 2) + 0 * x * p  # noqa: E731
    q = fw().WignerMoyalFTTW1D(**kw, V=lambda _, x: V(x), K=lambda _, p: 0.5 * p * p,
                               diff_V=lambda _, x: 0.2 * x ** 3 - 2 * x, diff_K=lambda _, p: p, precision="float32")
    q.set_wignerfunction(lambda _, x, p: init(x, p))
    W = q.propagate(20)
    o = WignerOracle(**kw, V=V, K=lambda p: 0.5 * p * p, diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p)
    o.set_wignerfunction(init(o.X, o.P))
    o.propagate(20)
    assert rel_l2(W, o.W) < FP32_TOL
    for k in ("X_average", "P_average", "X_average_RHS"):
        rtol, atol = FP32_OBS_TOL[k]
        np.testing.assert_allclose(getattr(q, k), getattr(o, k), rtol=rtol, atol=atol)


def test_fp32_bloch_256():
    case = dict(CASES["bloch_fftw_harmonic_128"])
    kw = dict(case["kw"], X_gridDIM=256, P_gridDIM=256)
    q = fw().WignerBlochFFTW1D(**kw, precision="float32")
    W = q.get_gibbs_state()
    o = WignerOracle(**{k: v for k, v in kw.items() if k not in ("kT", "dbeta", "V", "K")},
                     V=lambda x: 0.5 * x ** 2, K=lambda p: 0.5 * p ** 2)
    o.setup_bloch_fftw(kw["kT"], kw["dbeta"])
    o.get_gibbs_state_fftw()
    assert rel_l2(W, o.W) < FP32_TOL


@pytest.mark.parametrize("P,X,precision", [(2048, 128, "float32"), (4096, 128, "float32"), (128, 4096, "float32"),
                                           (1024, 2048, "float32"),
                                           (1024, 128, "float64"), (2048, 128, "float64"), (4096, 128, "float64"),
                                           (128, 4096, "float64")])
def test_extreme_grid_shapes_match_oracle(P, X, precision):
    """The largest transform lengths on either axis (each column / row pass
    launch shape of the 2048- and 4096-point transforms; 1024 x 2048 is the
    strong-field grid, whose one-instance plan runs the small-batch row shape)
    against the FP64 oracle."""
    kw = dict(t=0.0, dt=0.005, X_gridDIM=X, X_amplitude=10.0, P_gridDIM=P, P_amplitude=10.0)
    V = lambda x: 0.05 * x ** 4 - x ** 2  # noqa: E731
    init = lambda x, p: np.exp(-(x + 1.3) ** 2 / 0.5 - 0.25 * (p - 0.4) ** 2) + 0 * x * p  # noqa: E731
    q = fw().WignerMoyalFTTW1D(**kw, V=lambda _, x: V(x), K=lambda _, p: 0.5 * p * p,
                               diff_V=lambda _, x: 0.2 * x ** 3 - 2 * x, diff_K=lambda _, p: p, precision=precision)
    q.set_wignerfunction(lambda _, x, p: init(x, p))
    W = q.propagate(10)
    o = WignerOracle(**kw, V=V, K=lambda p: 0.5 * p * p, diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p)
    o.set_wignerfunction(init(o.X, o.P))
    o.propagate(10)
    if precision == "float64":
        assert rel_l2(W, o.W) < FP64_TOL
        for k in ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average"):
            np.testing.assert_allclose(getattr(q, k), getattr(o, k), rtol=FP64_TOL, atol=FP64_TOL)
    else:
        assert rel_l2(W, o.W) < FP32_TOL
        for k in ("X_average", "P_average", "X_average_RHS"):
            rtol, atol = FP32_OBS_TOL[k]
            np.testing.assert_allclose(getattr(q, k), getattr(o, k), rtol=rtol, atol=atol)


def test_zero_steps_leave_the_state_alone():
    kw = dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0)
    q = fw().WignerMoyalFTTW1D(**kw, V=lambda _, x: 0.5 * x * x, K=lambda _, p: 0.5 * p * p,
                               diff_V=lambda _, x: x, diff_K=lambda _, p: p)
    q.set_wignerfunction(lambda _, x, p: np.exp(-(x - 1) ** 2 - (p - 0.5) ** 2) + 0 * x * p)
    W0 = np.array(q.wignerfunction, copy=True)
    n0 = len(q.X_average)
    W = q.propagate(0)
    np.testing.assert_array_equal(np.asarray(W), W0)
    assert q.t == 0.0 and len(q.X_average) == n0
