"""Parity of the exact plan that bench.py times, and of the 1024 x 1024
double-well configuration at its full length, against the FP64 oracle.

The bench plan is ``WignerMoyalBatch`` on the 1024 x 1024 double well
(V = 0.05 x^4 - x^2, amplitudes 10/10, dt = 0.005, Gaussian packets with
x0 ~ U(-2, 2), p0 ~ U(-1, 1), width 0.5), FP32 state, 8 observables per
instance.  A batch of 8 already takes every code path of the 64-instance
bench launch: the regular launch shapes (8 x 64 column tiles >= the SM
count), the per-instance totals kernel (batch >= 4), the vector loads of the
shared phase table (tab_vec) and the fused mid-point column pass with its
p-weight spectra.  A batch of 16 adds the persistent row pass.  Every instance
is compared with the oracle restatement of WignerMoyalFTTW1D.propagate
(wigner_moyal_fftw_1d.py:418-440).

Tolerances (tests/parity_tables.py): FP64 1e-10 relative on W and every
observable; FP32 1e-5 relative L2 of W for a short run, and for long runs
within PIPELINE_FACTOR x the error of a plain complex64 pipeline on the same
input (the FP32 error of any FFT pipeline grows linearly with the steps)."""
import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests"))
import bench  # noqa: E402
from oracle.wigner_oracle import WignerOracle  # noqa: E402
from parity_tables import (_errors, complex64_pipeline, config2_error_table, ehrenfest_from_sums,  # noqa: E402
                           within_pipeline)

pytestmark = pytest.mark.gpu
OBS = ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average")


def _oracle(W0):
    o = WignerOracle(X_gridDIM=bench.GRID, X_amplitude=bench.AMP, P_gridDIM=bench.GRID, P_amplitude=bench.AMP,
                     dt=bench.DT, V=bench.V, K=bench.K, diff_V=bench.dV, diff_K=bench.dK,
                     fft_workers=os.cpu_count())
    o.cache_exponents()
    o.set_wignerfunction(np.asarray(W0, dtype=np.float64))
    return o


def _bench_plan(batch, precision, steps, seed):
    import torch

    from fastwigner_b200.batch import WignerMoyalBatch

    sim = WignerMoyalBatch(batch=batch, X_gridDIM=bench.GRID, X_amplitude=bench.AMP, P_gridDIM=bench.GRID,
                           P_amplitude=bench.AMP, dt=bench.DT, V=bench.V, K=bench.K, diff_V=bench.dV,
                           diff_K=bench.dK, precision=precision)
    W0 = bench.initial_states(np.random.default_rng(seed), batch, sim.X, sim.P)
    sim.set_wignerfunctions(torch.from_numpy(W0).cuda())
    W0n = sim.W.double().cpu().numpy()  # the normalised start states, as the oracle sees them
    obs = sim.propagate(steps).cpu().numpy()
    torch.cuda.synchronize()
    return sim, W0n, obs


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision,steps", [("float32", 200), ("float64", 40)])
def test_bench_plan_matches_oracle_every_instance(precision, steps):
    """FP64: 1e-10 on W and every observable.  FP32 over 200 steps: within
    PIPELINE_FACTOR x the error a plain complex64 pipeline makes on the same
    instance (the FP32 error grows linearly with the steps; see
    tests/parity_tables.py), and never above 1e-4 relative L2 of W."""
    batch = 8
    sim, W0n, obs = _bench_plan(batch, precision, steps, seed=2024)
    W = sim.W.double().cpu().numpy()
    for b in range(batch):
        o = _oracle(W0n[b])
        o.propagate(steps)
        got = ehrenfest_from_sums(obs[:, b, :])
        if precision == "float64":
            assert _rel(W[b], o.W) < 1e-10, b
            for k in OBS:
                np.testing.assert_allclose(got[k], getattr(o, k), rtol=1e-10, atol=1e-12, err_msg=f"{k} {b}")
        else:
            ours = _errors(got, o, W[b], o.W)
            Wc, oc = complex64_pipeline(W0n[b], steps, grid=bench.GRID, amp=bench.AMP, dt=bench.DT, V=bench.V,
                                        K=bench.K, dV=bench.dV, dK=bench.dK)
            pipe = _errors(oc, o, Wc, o.W)
            bad = within_pipeline(ours, pipe)
            assert not bad, (b, bad)
            assert ours["W_rel_l2"] < 1e-4, b
        # the per-step norm sums the plan records are the un-normalised sums of a normalised state
        assert np.allclose(obs[:, b, 0] * sim.dXdP, 1.0, atol=1e-4 if precision == "float32" else 1e-10)


def test_bench_plan_short_run_meets_the_fixed_fp32_tolerance():
    """20 steps of the FP32 bench plan (the bench line's own parity check):
    1e-5 relative L2 of W."""
    steps = 20
    sim, W0n, obs = _bench_plan(8, "float32", steps, seed=7)
    W = sim.W.double().cpu().numpy()
    for b in (0, 7):
        o = _oracle(W0n[b])
        o.propagate(steps)
        assert _rel(W[b], o.W) < 1e-5, b


def test_bench_plan_batch16_persistent_row_pass():
    """A batch of 16 (16 x 512 row pairs: enough work for the persistent row
    pass, which a batch of 8 leaves to the regular row kernel; both persistent
    passes and the call's single half-steps then run) against the oracle over
    20 FP32 steps at 1e-5, the first and the last instance (whose last row
    pair ends the state buffer)."""
    steps = 20
    sim, W0n, obs = _bench_plan(16, "float32", steps, seed=11)
    W = sim.W.double().cpu().numpy()
    for b in (0, 15):
        o = _oracle(W0n[b])
        o.propagate(steps)
        assert _rel(W[b], o.W) < 1e-5, b


def test_config2_full_length_error_table():
    """One instance of the 1024 x 1024 double well through the drop-in class
    for the configuration's full 4000 steps, FP32 and FP64, against the FP64
    oracle: the error of every observable and of W.  FP64 within 1e-10; FP32
    within PIPELINE_FACTOR x the plain complex64 pipeline's error on the same
    run.  When FW_PARITY_TABLE names a file, the measured table is written
    there as JSON."""
    table = config2_error_table(steps=4000)
    out = os.environ.get("FW_PARITY_TABLE")
    if out:
        Path(out).write_text(json.dumps(table, indent=1))
    f32, f64, pipe = table["float32"], table["float64"], table["complex64_pipeline"]
    assert f64["W_rel_l2"] < 1e-10
    for k in OBS:
        assert f64["obs"][k]["max_abs"] <= 1e-10 * max(1.0, f64["obs"][k]["max_ref"]), k
    bad = within_pipeline(f32, pipe)
    assert not bad, bad


def test_per_instance_tables_batch_matches_oracle():
    """A 1024 x 1024 FP32 batch whose instances carry their own double wells
    (one phase table per instance: the column pass fetches a table tile per
    work item) against the oracle, 20 steps, 1e-5 relative L2 per instance."""
    import torch

    from fastwigner_b200.batch import WignerMoyalBatch

    B, steps = 8, 20
    rng = np.random.default_rng(31)
    ab = [(rng.uniform(0.02, 0.1), rng.uniform(0.5, 2.0)) for _ in range(B)]
    Vs = [(lambda a, b: (lambda x: a * x ** 4 - b * x ** 2))(a, b) for a, b in ab]
    Ks = [bench.K] * B
    sim = WignerMoyalBatch(batch=B, X_gridDIM=bench.GRID, X_amplitude=bench.AMP, P_gridDIM=bench.GRID,
                           P_amplitude=bench.AMP, dt=bench.DT, V=Vs, K=Ks, precision="float32", observables=False)
    W0 = bench.initial_states(rng, B, sim.X, sim.P)
    sim.set_wignerfunctions(torch.from_numpy(W0).cuda())
    W0n = sim.W.double().cpu().numpy()
    sim.propagate(steps)
    torch.cuda.synchronize()
    W = sim.W.double().cpu().numpy()
    for b in range(B):
        o = WignerOracle(X_gridDIM=bench.GRID, X_amplitude=bench.AMP, P_gridDIM=bench.GRID, P_amplitude=bench.AMP,
                         dt=bench.DT, V=Vs[b], K=bench.K, fft_workers=os.cpu_count())
        o.cache_exponents()
        o.set_wignerfunction(W0n[b])
        o.propagate(steps)
        assert _rel(W[b], o.W) < 1e-5, b
