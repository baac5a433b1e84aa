"""Batched propagation: uniform batches (one launch per pass, batch in grid.y)
and uneven batches (one persistent cooperative launch) against single-instance
runs and the FP64 oracle."""
import numpy as np
import pytest

from oracle.wigner_oracle import WignerOracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def dw(a, b):
    return (lambda x: a * x ** 4 - b * x ** 2), (lambda p: 0.5 * p ** 2)


SIZES = [(128, 256), (256, 128), (512, 512), (1024, 256), (128, 128), (256, 1024), (1024, 1024)]


def make_specs(rng):
    specs = []
    for P, X in SIZES:
        V, K = dw(rng.uniform(0.02, 0.1), rng.uniform(0.5, 2.0))
        specs.append(dict(P_gridDIM=P, X_gridDIM=X, X_amplitude=rng.uniform(6, 10), P_amplitude=rng.uniform(6, 10),
                          V=V, K=K))
    return specs


def initial(s, rng):
    x0, p0 = rng.uniform(-2, 2), rng.uniform(-1, 1)
    return (np.exp(-(s["X"] - x0) ** 2 / 0.25 - 0.25 * (s["P"] - p0) ** 2) + 0 * s["X"] * s["P"]).astype(np.float32)


@pytest.mark.parametrize("variant", [0, 1, "grouped"])
def test_uneven_batch_matches_oracle(variant):
    from fastwigner_b200.batch import WignerMoyalUnevenBatch

    rng = np.random.default_rng(3)
    specs = make_specs(rng)
    b = WignerMoyalUnevenBatch(specs, dt=0.005, variant=0)
    b.set_variant(b.GROUPED if variant == "grouped" else variant)
    states = [initial(s, rng) for s in b.specs]
    b.set_wignerfunctions(states)
    obs = b.propagate(25, use_graph=False)
    assert b.status() == 0
    for s, W0, W in zip(b.specs, states, b.W):
        o = WignerOracle(X_gridDIM=s["X_gridDIM"], X_amplitude=s["X_amplitude"], P_gridDIM=s["P_gridDIM"],
                         P_amplitude=s["P_amplitude"], dt=0.005, V=s["V"], K=s["K"])
        o.set_wignerfunction(W0.astype(np.float64))
        o.propagate(25)
        assert rel(W.double().cpu().numpy(), o.W) < 1e-5
    pur = b.purity(obs)
    assert np.all(np.isfinite(pur)) and np.all(pur <= 1.0 + 1e-4)


def test_graph_replay_equals_direct_launch_and_autotune_cache(tmp_path, monkeypatch):
    from fastwigner_b200.batch import WignerMoyalUnevenBatch

    monkeypatch.setenv("FASTWIGNER_AUTOTUNE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(5)
    specs = make_specs(rng)
    a = WignerMoyalUnevenBatch(specs, dt=0.005, variant=None, autotune_steps=3)
    assert (tmp_path / "tune.json").exists()
    b = WignerMoyalUnevenBatch(specs, dt=0.005, variant=a.variant)
    states = [initial(s, rng) for s in a.specs]
    a.set_wignerfunctions(states)
    b.set_wignerfunctions(states)
    for _ in range(3):
        a.propagate(10, use_graph=True)
        b.propagate(10, use_graph=False)
    for Wa, Wb in zip(a.W, b.W):  # same work per item whichever CTA takes it: bit-identical
        assert np.array_equal(Wa.cpu().numpy(), Wb.cpu().numpy())


def test_grouped_mode_equals_persistent_kernel_on_shared_shapes():
    """Instances of one shape and box share a plan in the grouped mode: six
    1024^2 instances (enough column pairs for the persistent pass kernels),
    three 256 x 512 and two 128^2, interleaved, each with its own potential.
    The grouped mode (graph replay after a direct first call) agrees with the
    persistent cooperative kernel and, for one instance per shape, with the
    oracle; graph replays equal direct launches bit for bit."""
    from fastwigner_b200.batch import WignerMoyalUnevenBatch

    rng = np.random.default_rng(9)
    shapes = [(1024, 1024), (256, 512), (1024, 1024), (128, 128), (1024, 1024), (256, 512),
              (1024, 1024), (128, 128), (1024, 1024), (256, 512), (1024, 1024)]
    specs = []
    for P, X in shapes:
        V, K = dw(rng.uniform(0.02, 0.1), rng.uniform(0.5, 2.0))
        specs.append(dict(P_gridDIM=P, X_gridDIM=X, X_amplitude=8.0, P_amplitude=7.0, V=V, K=K))
    a = WignerMoyalUnevenBatch(specs, dt=0.005, variant=0)
    b = WignerMoyalUnevenBatch(specs, dt=0.005, variant=0)
    c = WignerMoyalUnevenBatch(specs, dt=0.005, variant=0)
    b.set_variant(b.GROUPED)
    c.set_variant(c.GROUPED)
    assert len(b._groups) == 3
    states = [initial(s, rng) for s in a.specs]
    for x in (a, b, c):
        x.set_wignerfunctions(states)
    import torch

    ob = torch.empty((10, len(specs), 2), dtype=torch.float64, device="cuda")
    for _ in range(3):  # b: a direct call that captures the graph, then two replays
        oa = a.propagate(10, use_graph=False)
        b.propagate(10, use_graph=True, obs=ob)
        c.propagate(10, use_graph=False)
    assert a.status() == 0 and b.status() == 0 and c.status() == 0
    for Wa, Wb, Wc in zip(a.W, b.W, c.W):
        assert rel(Wb.double().cpu().numpy(), Wa.double().cpu().numpy()) < 1e-5
        assert np.array_equal(Wb.cpu().numpy(), Wc.cpu().numpy())
    np.testing.assert_allclose(b.purity(ob), a.purity(oa), rtol=1e-5)
    for i in (0, 1, 3):
        s = a.specs[i]
        o = WignerOracle(X_gridDIM=s["X_gridDIM"], X_amplitude=8.0, P_gridDIM=s["P_gridDIM"], P_amplitude=7.0,
                         dt=0.005, V=s["V"], K=s["K"])
        o.set_wignerfunction(states[i].astype(np.float64))
        o.propagate(30)
        assert rel(b.W[i].double().cpu().numpy(), o.W) < 1e-5


@pytest.mark.parametrize("B", [3, 12])
def test_uniform_batch_equals_single_instances(B):
    """FP64 256^2: a batch of 3 runs the small-batch launch shapes like the single
    instances; a batch of 12 (192 column CTAs, more than the SMs) the regular ones,
    so the two shape sets are checked against each other."""
    from fastwigner_b200 import WignerMoyalFTTW1D
    from fastwigner_b200.batch import WignerMoyalBatch

    V, K = dw(0.05, 1.0)
    kw = dict(X_gridDIM=256, X_amplitude=10.0, P_gridDIM=256, P_amplitude=10.0, dt=0.005)
    b = WignerMoyalBatch(batch=B, **kw, V=V, K=K, diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p,
                         precision="float64")
    rng = np.random.default_rng(1)
    W0 = np.stack([np.exp(-(b.X - rng.uniform(-2, 2)) ** 2 - (b.P - rng.uniform(-1, 1)) ** 2) for _ in range(B)])
    b.set_wignerfunctions(W0)
    obs = b.propagate(12).cpu().numpy()
    for i in range(B):
        q = WignerMoyalFTTW1D(**kw, t=0.0, V=lambda _, x: V(x), K=lambda _, p: K(p),
                              diff_V=lambda _, x: 0.2 * x ** 3 - 2 * x, diff_K=lambda _, p: p)
        q.set_wignerfunction(W0[i])
        W = q.propagate(12)
        assert rel(b.W[i].cpu().numpy(), W) < 1e-12
        np.testing.assert_allclose(obs[:, i, 2] / obs[:, i, 0], q.X_average, rtol=1e-11)


def test_host_batches_pipeline_equals_sequential_calls():
    """propagate_host_batches (copies on their own streams, two alternating
    device buffers) gives bit-identical states and observables to one
    set_wignerfunctions + propagate call per host batch."""
    import torch

    from fastwigner_b200.batch import WignerMoyalBatch

    V, K = dw(0.05, 1.0)
    kw = dict(X_gridDIM=256, X_amplitude=10.0, P_gridDIM=256, P_amplitude=10.0, dt=0.005, V=V, K=K,
              diff_V=lambda x: 0.2 * x ** 3 - 2 * x, diff_K=lambda p: p, precision="float32")
    B, n, steps = 4, 5, 20
    rng = np.random.default_rng(3)
    a = WignerMoyalBatch(batch=B, **kw)
    states = []
    for _ in range(n):
        W0 = np.stack([np.exp(-(a.X - rng.uniform(-2, 2)) ** 2 - (a.P - rng.uniform(-1, 1)) ** 2)
                       for _ in range(B)]).astype(np.float32)
        states.append(torch.from_numpy(W0).pin_memory())
    obs_out = [torch.empty((steps, B, 8), dtype=torch.float64).pin_memory() for _ in range(n)]
    out, _ = a.propagate_host_batches(states, steps, obs_out=obs_out)
    torch.cuda.synchronize()
    assert abs(a.t - steps * 0.005) < 1e-15
    b = WignerMoyalBatch(batch=B, **kw)
    for i in range(n):
        b.set_wignerfunctions(states[i].cuda())
        ob = b.propagate(steps)
        np.testing.assert_array_equal(out[i].numpy(), b.W.cpu().numpy())
        np.testing.assert_array_equal(obs_out[i].numpy(), ob.cpu().numpy())
    np.testing.assert_array_equal(a.W.cpu().numpy(), out[-1].numpy())


FW_BATCH_TIMEOUT = 1


def _oracle_states(b, states, steps):
    out = []
    for s, W0 in zip(b.specs, states):
        o = WignerOracle(X_gridDIM=s["X_gridDIM"], X_amplitude=s["X_amplitude"], P_gridDIM=s["P_gridDIM"],
                         P_amplitude=s["P_amplitude"], dt=0.005, V=s["V"], K=s["K"])
        o.set_wignerfunction(W0.astype(np.float64))
        o.propagate(steps)
        out.append(o.W)
    return out


def test_planted_status_makes_the_launch_return_early_and_clears():
    """A non-zero status word planted from the host before the launch: every
    CTA reads it at the first grid barrier and returns, the word still reads
    FW_BATCH_TIMEOUT afterwards, and once it is cleared the same batch runs
    normally (the context stays usable).  No wait is left unbounded."""
    import torch

    from fastwigner_b200.batch import WignerMoyalUnevenBatch

    rng = np.random.default_rng(8)
    b = WignerMoyalUnevenBatch(make_specs(rng), dt=0.005, variant=0)
    states = [initial(s, rng) for s in b.specs]
    b.set_wignerfunctions(states)
    b.set_status(FW_BATCH_TIMEOUT)
    b.propagate(2, use_graph=False)
    torch.cuda.synchronize()
    assert b.status() == FW_BATCH_TIMEOUT
    b.set_status(0)
    b.set_wignerfunctions(states)
    b.t = 0.0
    b.propagate(2, use_graph=False)
    torch.cuda.synchronize()
    assert b.status() == 0
    for W, ref in zip(b.W, _oracle_states(b, states, 2)):
        assert rel(W.double().cpu().numpy(), ref) < 1e-5


def test_barrier_wait_limit_expires_and_returns():
    """A spin limit of 0 polls: the first CTA that has to wait at a grid
    barrier gives up at once and records FW_BATCH_TIMEOUT, the others see the
    word and return, and the launch ends.  Afterwards (limit restored, word
    cleared) the batch propagates correctly."""
    import torch

    from fastwigner_b200.batch import WignerMoyalUnevenBatch

    rng = np.random.default_rng(9)
    b = WignerMoyalUnevenBatch(make_specs(rng), dt=0.005, variant=0)
    states = [initial(s, rng) for s in b.specs]
    b.set_spin_limit(0)
    seen = 0
    for _ in range(3):  # the first arriver could in principle find the barrier already released
        b.set_status(0)
        b.set_wignerfunctions(states)
        b.propagate(2, use_graph=False)
        torch.cuda.synchronize()
        seen = b.status()
        if seen == FW_BATCH_TIMEOUT:
            break
    assert seen == FW_BATCH_TIMEOUT
    b.set_spin_limit(1 << 25)
    b.set_status(0)
    b.set_wignerfunctions(states)
    b.t = 0.0
    b.propagate(2, use_graph=True)
    torch.cuda.synchronize()
    assert b.status() == 0
    for W, ref in zip(b.W, _oracle_states(b, states, 2)):
        assert rel(W.double().cpu().numpy(), ref) < 1e-5
