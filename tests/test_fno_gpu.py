"""FNO surrogate kernels on the GPU: forward output and every parameter
gradient against the FP64 numpy oracle, and a short training run.
Tolerances: forward 1e-4 relative L2, gradients 2e-3 relative L2 (FP32 kernels,
FP64 oracle)."""
import numpy as np
import pytest
import torch

from oracle.fno_oracle import FNOOracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30)


def test_forward_and_gradients_match_oracle():
    from fastwigner_b200.fno import FNO2d

    net = FNO2d(n_params=3, width=8, modes=(4, 5), layers=3, proj=16, seed=3)
    # larger spectral weights than the default init so every path matters
    for l in range(3):
        net.params[f"R{l}"].mul_(20.0)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(3, 3))
    xs = np.linspace(-1, 1, 32, endpoint=False)
    ps = np.linspace(-1, 1, 24, endpoint=False)
    T = rng.normal(size=(3, 24, 32))
    y = net.forward(X, xs, ps).double().cpu().numpy()
    o = FNOOracle({k: v.double().cpu().numpy() for k, v in net.params.items()}, 3, 8, (4, 5), 3, 16)
    yo = o.forward(X, xs, ps)
    assert rel(y, yo) < 1e-4
    dY = torch.tensor(yo - T, dtype=torch.float32, device="cuda")
    g = net.backward(dY)
    go = o.backward(yo - T)
    for k in net.names:
        assert rel(g[k].double().cpu().numpy(), go[k]) < 2e-3, k


def test_inference_path_equals_training_path():
    """forward(cache=False) (no stored activations, the fused projection with
    the 128-wide hidden layer kept in tensor memory) against forward(cache=True)
    (pre-activations stored, unfused projection) and the FP64 oracle."""
    from fastwigner_b200.fno import FNO2d

    net = FNO2d(n_params=3, width=32, modes=(8, 8), layers=4, proj=128, seed=5)
    for l in range(4):
        net.params[f"R{l}"].mul_(20.0)
    rng = np.random.default_rng(2)
    X = rng.normal(size=(5, 3))
    xs = np.linspace(-1, 1, 96, endpoint=False)
    ps = np.linspace(-1, 1, 64, endpoint=False)
    a = net.forward(X, xs, ps, cache=True).double().cpu().numpy()
    b = net.forward(X, xs, ps, cache=False).double().cpu().numpy()
    assert rel(b, a) < 1e-5
    o = FNOOracle({k: v.double().cpu().numpy() for k, v in net.params.items()}, 3, 32, (8, 8), 4, 128)
    assert rel(b, o.forward(X, xs, ps)) < 1e-4


def test_training_reduces_loss():
    from fastwigner_b200.fno import FNO2d

    net = FNO2d(n_params=3, width=16, modes=(6, 6), layers=2, proj=32, seed=1)
    rng = np.random.default_rng(1)
    xs = np.linspace(-1, 1, 32, endpoint=False).astype(np.float32)
    ps = np.linspace(-1, 1, 32, endpoint=False).astype(np.float32)
    X = rng.uniform(-1, 1, size=(64, 3))
    # smooth parametric targets: shifted, squeezed Gaussians
    T = np.exp(-((xs[None, None, :] - 0.4 * X[:, 0, None, None]) ** 2) / (0.2 + 0.1 * X[:, 1, None, None]) ** 2
               - ((ps[None, :, None] - 0.3 * X[:, 2, None, None]) ** 2) / 0.3)
    T = torch.tensor(T, dtype=torch.float32, device="cuda")
    first = last = None
    for it in range(300):
        idx = rng.choice(64, size=16, replace=False)
        loss, dY = net.loss_and_grad(X[idx], xs, ps, T[torch.as_tensor(idx)])
        net.backward(dY)
        net.adam_step(3e-3)
        first = loss if first is None else first
        last = loss
    assert last < 0.1 * first, (first, last)


def test_trained_surrogate_gains_over_the_plain_bloch_run():
    """What the trained network buys: a small FNO trained on plain-Bloch Morse
    trajectories seeds the Bloch run at beta_s = 0.8 beta; the refined state
    is far closer to the plain thermal state than the plain run given the
    same number of Bloch steps, with at most a quarter of the plain steps,
    and the network seed refines better than its analytic harmonic baseline
    alone."""
    from fastwigner_b200.fno import BlochBatch, BlochSurrogate, FNO2d, MorseBlochSetup, generate_dataset

    setup = MorseBlochSetup(grid=128, X_amplitude=8.0, P_amplitude=8.0, dbeta=2e-3)
    rng = np.random.default_rng(0)
    betas = np.exp(np.linspace(np.log(0.2), np.log(6.0), 24))
    P, S = generate_dataset(setup, 48, betas, rng, train_grid=64)
    net = FNO2d(n_params=3, width=16, modes=(8, 8), layers=3, proj=64, seed=0)
    sur = BlochSurrogate(setup, net, train_grid=64)
    sur.train(P, S, epochs=8, batch=16, rng=rng)

    Ds, As, beta = rng.uniform(2.0, 10.0, 4), rng.uniform(0.5, 1.5, 4), 5.0
    dxdp = setup.dX * setup.dP
    bb = BlochBatch(setup, Ds, As)
    Wp, n_plain = sur.plain_gibbs(bb, beta)
    Wp = Wp.clone()

    def err(W):
        return float(((W - Wp).abs().amax(dim=(1, 2)).double() * dxdp).max())

    Ws, n_seed = sur.seeded_gibbs(bb, Ds, As, beta, refine_fraction=0.2, min_refine=0.5)
    e_seed = err(Ws)
    e_plain_same = err(bb.set_uniform().run(n_seed).W)  # the method without the network, same steps
    bs = beta - n_seed * setup.dbeta
    B = sur.baseline(np.stack([Ds, As, np.full(4, bs)], axis=1))
    e_base = err(bb.set_states(B).run(n_seed).W)  # the analytic seed alone, same steps
    assert n_seed <= 0.25 * n_plain
    assert e_seed < 0.05 * e_plain_same, (e_seed, e_plain_same)
    assert e_seed < e_base, (e_seed, e_base)
