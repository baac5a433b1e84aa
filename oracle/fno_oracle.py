"""FP64 numpy oracle of the FNO surrogate (forward and backward).

TEST INFRASTRUCTURE ONLY: checks the GPU kernels' forward output and
parameter gradients (tests/test_fno_gpu.py), and is itself checked against
central finite differences (tests/test_fno_oracle.py).  The network has no
reference counterpart; this restates the architecture of
fastwigner_b200/fno.py in plain numpy.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

from fastwigner_b200.fno import dft_matrices


def gelu(x):
    return 0.5 * x * (1 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


class FNOOracle:
    def __init__(self, params: dict, n_params, width, modes, layers, proj):
        self.p = {k: np.asarray(v, dtype=np.float64) for k, v in params.items()}
        self.NP, self.C, self.mp, self.mx, self.layers, self.proj = n_params, width, modes[0], modes[1], layers, proj
        self.Kp = 2 * self.mp
        self.K = self.Kp * self.mx

    def _mix(self, F, R):  # F (B, C, 2, K), R (C, C, 2, K)
        Fc = F[:, :, 0] + 1j * F[:, :, 1]
        Rc = R[:, :, 0] + 1j * R[:, :, 1]
        O = np.einsum("bik,iok->bok", Fc, Rc)
        return np.stack([O.real, O.imag], axis=2)

    def forward(self, X, xs, ps):
        """X (B, NP) normalised inputs.  Returns (B, G0, G1) and the cache."""
        p, C, NP = self.p, self.C, self.NP
        B, G0, G1 = len(X), len(ps), len(xs)
        L = G0 * G1
        Cx, Sx, Dp, Dpi, A1, A2 = dft_matrices(G0, G1, self.mp, self.mx)
        feats = np.empty((B, NP + 2, G0, G1))
        feats[:, :NP] = X[:, :, None, None]
        feats[:, NP] = xs[None, None, :]
        feats[:, NP + 1] = ps[None, :, None]
        v = np.einsum("oi,bil->bol", p["W0"], feats.reshape(B, NP + 2, L)) + p["b0"][None, :, None]
        cache = {"feats": feats.reshape(B, NP + 2, L), "v": [], "F2": [], "pre": []}
        for l in range(self.layers):
            cache["v"].append(v)
            V = v.reshape(B, C, G0, G1)
            Fx2 = np.concatenate([V @ Cx, V @ Sx], axis=2)                       # (B, C, 2G0, mx)
            F2 = (Dp @ Fx2).reshape(B, C, 2, self.K)                              # (B, C, 2Kp, mx)
            cache["F2"].append(F2)
            O2 = self._mix(F2, p[f"R{l}"]).reshape(B, C, 2 * self.Kp, self.mx)
            Gx2 = Dpi @ O2                                                        # (B, C, 2G0, mx)
            y = Gx2[:, :, :G0] @ A1 + Gx2[:, :, G0:] @ A2                        # (B, C, G0, G1)
            y = y.reshape(B, C, L) + np.einsum("oi,bil->bol", p[f"W{l + 1}"], v)
            pre = y + p[f"b{l + 1}"][None, :, None]
            cache["pre"].append(pre)
            v = gelu(pre) if l < self.layers - 1 else pre
        cache["vL"] = v
        pre1 = np.einsum("oi,bil->bol", p["Q1"], v) + p["c1"][None, :, None]
        a1 = gelu(pre1)
        out = np.einsum("oi,bil->bol", p["Q2"], a1) + p["c2"][None, :, None]
        cache.update(pre1=pre1, a1=a1, dims=(B, G0, G1))
        self.cache = cache
        return out.reshape(B, G0, G1)

    def backward(self, dout):
        c, p, C, NP = self.cache, self.p, self.C, self.NP
        B, G0, G1 = c["dims"]
        L = G0 * G1
        Cx, Sx, Dp, Dpi, A1, A2 = dft_matrices(G0, G1, self.mp, self.mx)
        g = {}
        d = dout.reshape(B, 1, L)
        g["c2"] = d.sum(axis=(0, 2))
        g["Q2"] = np.einsum("bol,bil->oi", d, c["a1"])
        da1 = np.einsum("oi,bol->bil", p["Q2"], d) * gelu_d(c["pre1"])
        g["c1"] = da1.sum(axis=(0, 2))
        g["Q1"] = np.einsum("bol,bil->oi", da1, c["vL"])
        dv = np.einsum("oi,bol->bil", p["Q1"], da1)
        for l in reversed(range(self.layers)):
            dpre = dv * gelu_d(c["pre"][l]) if l < self.layers - 1 else dv
            g[f"b{l + 1}"] = dpre.sum(axis=(0, 2))
            vin = c["v"][l]
            g[f"W{l + 1}"] = np.einsum("bol,bil->oi", dpre, vin)
            dvin = np.einsum("oi,bol->bil", p[f"W{l + 1}"], dpre)
            D4 = dpre.reshape(B, C, G0, G1)
            dGx2 = np.concatenate([D4 @ A1.T, D4 @ A2.T], axis=2)
            dO2 = (Dpi.T @ dGx2).reshape(B, C, 2, self.K)
            dOc = dO2[:, :, 0] + 1j * dO2[:, :, 1]
            R = p[f"R{l}"]
            Rc = R[:, :, 0] + 1j * R[:, :, 1]
            dFc = np.einsum("bok,iok->bik", dOc, np.conj(Rc))
            F2 = c["F2"][l]
            Fc = F2[:, :, 0] + 1j * F2[:, :, 1]
            dRc = np.einsum("bik,bok->iok", np.conj(Fc), dOc)
            g[f"R{l}"] = np.stack([dRc.real, dRc.imag], axis=2)
            dF2 = np.stack([dFc.real, dFc.imag], axis=2).reshape(B, C, 2 * self.Kp, self.mx)
            dFx2 = Dp.T @ dF2
            dvin = dvin + (dFx2[:, :, :G0] @ Cx.T + dFx2[:, :, G0:] @ Sx.T).reshape(B, C, L)
            dv = dvin
        g["b0"] = dv.sum(axis=(0, 2))
        g["W0"] = np.einsum("bol,bil->oi", dv, c["feats"])
        return g
