"""Pin the numpy FNO oracle's backward pass with central finite differences (CPU)."""
import numpy as np

from oracle.fno_oracle import FNOOracle


def tiny(seed=0):
    rng = np.random.default_rng(seed)
    C, NP, K, PJ, L = 3, 3, 2 * 2 * 3, 5, 2
    p = {"W0": rng.normal(size=(C, NP + 2)) * 0.5, "b0": rng.normal(size=C) * 0.1,
         "Q1": rng.normal(size=(PJ, C)) * 0.5, "c1": rng.normal(size=PJ) * 0.1,
         "Q2": rng.normal(size=(1, PJ)) * 0.5, "c2": rng.normal(size=1) * 0.1}
    for l in range(L):
        p[f"R{l}"] = rng.normal(size=(C, C, 2, K)) * 0.3
        p[f"W{l + 1}"], p[f"b{l + 1}"] = rng.normal(size=(C, C)) * 0.5, rng.normal(size=C) * 0.1
    return FNOOracle(p, NP, C, (2, 3), L, PJ), rng


def test_oracle_backward_matches_finite_differences():
    o, rng = tiny()
    X = rng.normal(size=(2, 3))
    xs, ps = np.linspace(-1, 1, 8, endpoint=False), np.linspace(-1, 1, 8, endpoint=False)
    T = rng.normal(size=(2, 8, 8))

    def loss():
        y = o.forward(X, xs, ps)
        return 0.5 * np.sum((y - T) ** 2)

    y = o.forward(X, xs, ps)
    g = o.backward(y - T)
    for name in ["W0", "b0", "R0", "W1", "b2", "R1", "Q1", "c1", "Q2", "c2"]:
        a = o.p[name]
        flat = a.reshape(-1)
        for idx in rng.choice(flat.size, size=min(4, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + 1e-6
            lp = loss()
            flat[idx] = old - 1e-6
            lm = loss()
            flat[idx] = old
            fd = (lp - lm) / 2e-6
            assert abs(fd - g[name].reshape(-1)[idx]) <= 1e-5 * max(1.0, abs(fd)), name
