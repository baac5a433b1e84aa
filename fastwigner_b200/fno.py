"""Fourier neural operator (FNO) surrogate for Bloch thermal states.

Maps the parameters of a potential and the inverse temperature beta to the
thermal Wigner function W(x, p).  Architecture (Li et al., FNO): a pointwise
lift of [params, x, p] to `width` channels, `layers` Fourier layers
v <- GELU(K(v) + W v + b) (no GELU after the last), a two-layer pointwise
projection.  K keeps modes_p x modes_x low modes of the 2-D spectrum (both
signs along p, non-negative along x of the real input) and mixes channels per
mode with learned complex weights.

Every operation runs in libfastwigner's own CUDA kernels (fw_fno_*): the
truncated DFTs are products with DFT matrices (forward normalised by 1/G),
the channel maps and projection are tensor-core GEMMs, the spectral mixing,
bias + GELU, reductions, loss and Adam have dedicated kernels.  Backward
passes are written out by hand (no autograd).  The reference has no learned
component.

The network's coordinate features (x and p) are not periodic over the box,
so the truncated DFT coefficients of the activations depend on the sampling
grid: a network trained on a 256^2 subgrid differs from itself on the full
512^2 grid by 4-5 % of its maximum.  Train on the grid the surrogate is
evaluated on (BlochSurrogate's default).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._device import require_cuda, stream_handle
from ._lib import check

F32 = 4


def _p(t, off=0):
    return ctypes.c_void_p(t.data_ptr() + F32 * int(off))


class _Ops:
    def __init__(self):
        self.lib = _lib.load()
        self._work = None  # split-K slices of the weight gradients

    def gemm(self, ta, tb, M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, batch, alpha=1.0, beta=0.0, oA=0, oB=0,
             oC=0):
        check(self.lib.fw_fno_sgemm(ta, tb, M, N, K, alpha, _p(A, oA), lda, sA, _p(B, oB), ldb, sB, beta, _p(C, oC),
                                    ldc, sC, batch, stream_handle()), "fw_fno_sgemm")

    def gemm_ex(self, ta, tb, M, N, K, A, lda, sA, B, ldb, sB, out, ldc, sC, batch, alpha=1.0, beta=0.0, C=None,
                bias=None, pre=None, aux=None, act=0, oA=0, oB=0):
        """out = epilogue(alpha op(A) op(B) + beta C + bias[m]); pre (if given) = the
        pre-activation; act 0: none, 1: GELU, 2: times GELU'(aux)."""
        opt = lambda t: _p(t) if t is not None else None
        check(self.lib.fw_fno_sgemm_ex(ta, tb, M, N, K, alpha, _p(A, oA), lda, sA, _p(B, oB), ldb, sB, beta, opt(C),
                                       ldc, sC, batch, opt(bias), opt(pre), opt(aux), int(act), _p(out),
                                       stream_handle()), "fw_fno_sgemm_ex")

    def wgrad(self, rows, cols, L, dY, X, batch, out):
        """out[r][c] = sum_b sum_l dY[b][r][l] X[b][c][l] (split-K on the tensor cores)."""
        n = ctypes.c_longlong(0)
        check(self.lib.fw_fno_wgrad_work(rows, cols, L, batch, ctypes.byref(n)), "fw_fno_wgrad_work")
        if self._work is None or self._work.numel() < n.value:
            self._work = torch.empty(n.value, dtype=torch.float32, device=dY.device)
        check(self.lib.fw_fno_wgrad(rows, cols, L, _p(dY), rows * L, _p(X), cols * L, batch, _p(self._work),
                                    self._work.numel(), _p(out), 0, stream_handle()), "fw_fno_wgrad")

    def project(self, hidden, C, L, V, batch, Q1, c1, Q2, c2, out):
        check(self.lib.fw_fno_project(hidden, C, L, _p(V), C * L, batch, _p(Q1), _p(c1), _p(Q2), _p(c2), _p(out), L,
                                      stream_handle()), "fw_fno_project")

    def mix(self, mode, B, Ci, Co, K, X, Y, out):
        check(self.lib.fw_fno_mix(mode, B, Ci, Co, K, _p(X), _p(Y), _p(out), stream_handle()), "fw_fno_mix")

    def bias_act(self, X, C, L, bias, pre, Y, act):
        check(self.lib.fw_fno_bias_act(X.numel(), C, L, _p(X), _p(bias), _p(pre) if pre is not None else None,
                                       _p(Y), int(act), stream_handle()), "fw_fno_bias_act")

    def act_bwd(self, dY, pre, dpre, act):
        check(self.lib.fw_fno_act_bwd(dY.numel(), _p(dY), _p(pre), _p(dpre), int(act), stream_handle()),
              "fw_fno_act_bwd")

    def csum(self, B, C, L, X, out, acc=False):
        check(self.lib.fw_fno_channel_sum(B, C, L, _p(X), _p(out), int(acc), stream_handle()), "fw_fno_channel_sum")

    def rel_l2(self, B, L, Y, T, dY, loss):
        check(self.lib.fw_fno_rel_l2(B, L, _p(Y), _p(T), _p(dY) if dY is not None else None,
                                     ctypes.c_void_p(loss.data_ptr()), stream_handle()), "fw_fno_rel_l2")

    def adam(self, p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        check(self.lib.fw_fno_adam(p.numel(), _p(p), _p(g), _p(m), _p(v), lr, b1, b2, eps, step, wd,
                                   stream_handle()), "fw_fno_adam")

    def features(self, B, NP, G0, G1, params, xs, ps, out):
        check(self.lib.fw_fno_features(B, NP, G0, G1, _p(params), _p(xs), _p(ps), _p(out), stream_handle()),
              "fw_fno_features")


def dft_matrices(G0, G1, mp, mx):
    """Truncated forward / inverse DFT matrices (float64 numpy) for a G0 x G1 grid.
    Returns Cx, Sx (G1 x mx), Dp (2Kp x 2G0), Dpi (2G0 x 2Kp), A1, A2 (mx x G1)."""
    if 2 * mx > G1 or 2 * mp > G0:
        raise ValueError("retained modes must be below the Nyquist frequency of the grid")
    x = np.arange(G1)
    kx = np.arange(mx)
    ax = 2 * np.pi * np.outer(x, kx) / G1
    Cx, Sx = np.cos(ax) / G1, -np.sin(ax) / G1
    kp = np.concatenate([np.arange(mp), np.arange(G0 - mp, G0)])
    th = 2 * np.pi * np.outer(kp, np.arange(G0)) / G0  # Kp x G0
    c, s = np.cos(th) / G0, np.sin(th) / G0
    Dp = np.block([[c, s], [-s, c]])
    ci, si = np.cos(th).T, np.sin(th).T  # G0 x Kp
    Dpi = np.block([[ci, -si], [si, ci]])
    w = np.where(kx == 0, 1.0, 2.0)[:, None]
    ang = 2 * np.pi * np.outer(kx, x) / G1
    A1, A2 = w * np.cos(ang), -w * np.sin(ang)
    return Cx, Sx, Dp, Dpi, A1, A2


class FNO2d:
    """The surrogate network.  ``n_params`` scalar inputs per sample."""

    def __init__(self, n_params=3, width=32, modes=(16, 16), layers=4, proj=128, seed=0, device=None):
        self.device = device or require_cuda()
        self.NP, self.C, self.layers, self.proj = int(n_params), int(width), int(layers), int(proj)
        self.mp, self.mx = int(modes[0]), int(modes[1])
        self.Kp = 2 * self.mp
        self.K = self.Kp * self.mx
        rng = np.random.default_rng(seed)
        C, NI = self.C, self.NP + 2

        def lin(o, i):
            b = 1.0 / math.sqrt(i)
            return rng.uniform(-b, b, size=(o, i)), rng.uniform(-b, b, size=(o,))

        p = {}
        p["W0"], p["b0"] = lin(C, NI)
        for l in range(self.layers):
            p[f"R{l}"] = (1.0 / (C * C)) * rng.uniform(0, 1, size=(C, C, 2, self.K))
            p[f"W{l + 1}"], p[f"b{l + 1}"] = lin(C, C)
        p["Q1"], p["c1"] = lin(self.proj, C)
        p["Q2"], p["c2"] = lin(1, self.proj)
        self.names = list(p)
        self.params = {k: torch.tensor(v, dtype=torch.float32, device=self.device).contiguous() for k, v in p.items()}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step = 0
        self.ops = _Ops()
        self._mats = {}
        self.input_scale = np.ones(self.NP)
        self.input_shift = np.zeros(self.NP)

    # -- parameters -------------------------------------------------------------
    def state_dict(self):
        d = {k: v.cpu().numpy() for k, v in self.params.items()}
        d["__meta__"] = np.array([self.NP, self.C, self.mp, self.mx, self.layers, self.proj])
        d["__in_scale__"], d["__in_shift__"] = self.input_scale, self.input_shift
        return d

    def load_state_dict(self, d):
        for k in self.names:
            self.params[k].copy_(torch.as_tensor(np.asarray(d[k]), dtype=torch.float32))
        self.input_scale, self.input_shift = np.asarray(d["__in_scale__"]), np.asarray(d["__in_shift__"])

    def _grid(self, G0, G1):
        """The DFT matrices of dft_matrices in the layouts the GEMMs use: the x
        transform's cosine and sine parts side by side, CS = [Cx | Sx] (G1 x 2mx),
        so one product gives Fx = [v Cx | v Sx] (G0 x 2mx per channel); read as a
        2G0 x mx matrix its rows alternate cosine / sine parts, so the p transform
        takes Dp with its columns interleaved alike and the inverse Dpi with its
        rows interleaved; AA = [A1; A2] (2mx x G1) maps [Gc | Gs] back to x."""
        key = (G0, G1)
        if key not in self._mats:
            Cx, Sx, Dp, Dpi, A1, A2 = dft_matrices(G0, G1, self.mp, self.mx)
            Dpv = np.empty_like(Dp)
            Dpv[:, 0::2], Dpv[:, 1::2] = Dp[:, :G0], Dp[:, G0:]
            Dpiv = np.empty_like(Dpi)
            Dpiv[0::2], Dpiv[1::2] = Dpi[:G0], Dpi[G0:]
            mats = (np.concatenate([Cx, Sx], axis=1), Dpv, Dpiv, np.concatenate([A1, A2], axis=0))
            self._mats[key] = [torch.tensor(m, dtype=torch.float32, device=self.device).contiguous() for m in mats]
        return self._mats[key]

    # -- forward ------------------------------------------------------------------
    def forward(self, params, xs, ps, cache=True):
        """params: (B, NP) raw inputs; xs (G1,), ps (G0,) coordinates (already
        normalised to O(1)).  Returns (B, G0, G1).  With cache=False (inference)
        no activations are kept and the two-layer projection runs fused."""
        o = self.ops
        B = params.shape[0]
        G0, G1 = len(ps), len(xs)
        L = G0 * G1
        C, NP = self.C, self.NP
        CS, Dpv, Dpiv, AA = self._grid(G0, G1)
        dev = self.device
        pr = torch.tensor((np.asarray(params, dtype=np.float64) - self.input_shift) * self.input_scale,
                          dtype=torch.float32, device=dev).contiguous()
        xs_t = torch.tensor(np.asarray(xs), dtype=torch.float32, device=dev)
        ps_t = torch.tensor(np.asarray(ps), dtype=torch.float32, device=dev)
        feats = torch.empty((B, NP + 2, G0, G1), dtype=torch.float32, device=dev)
        o.features(B, NP, G0, G1, pr, xs_t, ps_t, feats)
        P = self.params
        v = torch.empty((B, C, G0, G1), dtype=torch.float32, device=dev)
        o.gemm_ex(0, 0, C, L, NP + 2, P["W0"], NP + 2, 0, feats, L, (NP + 2) * L, v, L, C * L, B, bias=P["b0"])
        c = {"B": B, "G0": G0, "G1": G1, "feats": feats, "v": [], "F2": [], "pre": []}
        Kp, mx, K = self.Kp, self.mx, self.K
        Fx = torch.empty((B * C, G0, 2 * mx), dtype=torch.float32, device=dev)
        Gx = torch.empty_like(Fx)
        for l in range(self.layers):
            if cache:
                c["v"].append(v)
            # truncated forward DFT: x (cosine and sine parts in one product), then p
            o.gemm(0, 0, G0, 2 * mx, G1, v, G1, L, CS, 2 * mx, 0, Fx, 2 * mx, 2 * G0 * mx, B * C)
            F2 = torch.empty((B, C, 2, K), dtype=torch.float32, device=dev)
            o.gemm(0, 0, 2 * Kp, mx, 2 * G0, Dpv, 2 * G0, 0, Fx, mx, 2 * G0 * mx, F2, mx, 2 * K, B * C)
            if cache:
                c["F2"].append(F2)
            O2 = torch.empty_like(F2)
            o.mix(0, B, C, C, K, F2, P[f"R{l}"], O2)
            # inverse p, then x (Hermitian weights)
            o.gemm(0, 0, 2 * G0, mx, 2 * Kp, Dpiv, 2 * Kp, 0, O2, mx, 2 * K, Gx, mx, 2 * G0 * mx, B * C)
            y = torch.empty((B, C, G0, G1), dtype=torch.float32, device=dev)
            o.gemm(0, 0, G0, G1, 2 * mx, Gx, 2 * mx, 2 * G0 * mx, AA, G1, 0, y, G1, L, B * C)
            # + pointwise channel map + bias, GELU (not after the last layer), in place
            act = l < self.layers - 1
            pre = torch.empty_like(y) if cache else None
            o.gemm_ex(0, 0, C, L, C, P[f"W{l + 1}"], C, 0, v, L, C * L, y, L, C * L, B, beta=1.0, C=y,
                      bias=P[f"b{l + 1}"], pre=pre, act=int(act))
            if cache:
                c["pre"].append(pre)
            v = y
        out = torch.empty((B, 1, G0, G1), dtype=torch.float32, device=dev)
        if not cache and self.proj <= 128:
            o.project(self.proj, C, L, v, B, P["Q1"], P["c1"], P["Q2"], P["c2"], out)
            return out.view(B, G0, G1)
        c["vL"] = v
        pre1 = torch.empty((B, self.proj, G0, G1), dtype=torch.float32, device=dev)
        a1 = torch.empty_like(pre1)
        o.gemm_ex(0, 0, self.proj, L, C, P["Q1"], C, 0, v, L, C * L, a1, L, self.proj * L, B, bias=P["c1"],
                  pre=pre1, act=1)
        o.gemm_ex(0, 0, 1, L, self.proj, P["Q2"], self.proj, 0, a1, L, self.proj * L, out, L, L, B, bias=P["c2"])
        c.update(pre1=pre1, a1=a1)
        if cache:
            self._cache = c
        return out.view(B, G0, G1)

    # -- backward -----------------------------------------------------------------
    def backward(self, dout):
        """Accumulate parameter gradients (self.grads, zeroed first) for
        d(loss)/d(output) = dout (B, G0, G1)."""
        o, c, P, g = self.ops, self._cache, self.params, self.grads
        for t in g.values():
            t.zero_()
        B, G0, G1 = c["B"], c["G0"], c["G1"]
        L, C, NP, Kp, mx, K, PJ = G0 * G1, self.C, self.NP, self.Kp, self.mx, self.K, self.proj
        CS, Dpv, Dpiv, AA = self._grid(G0, G1)
        dev = self.device
        d_out = dout.contiguous().view(B, 1, G0, G1)
        o.csum(B, 1, L, d_out, g["c2"])
        o.wgrad(1, PJ, L, d_out, c["a1"], B, g["Q2"])
        # da1 = GELU'(pre1) Q2^T d_out
        da1 = torch.empty((B, PJ, G0, G1), dtype=torch.float32, device=dev)
        o.gemm_ex(1, 0, PJ, L, 1, P["Q2"], PJ, 0, d_out, L, L, da1, L, PJ * L, B, aux=c["pre1"], act=2)
        o.csum(B, PJ, L, da1, g["c1"])
        o.wgrad(PJ, C, L, da1, c["vL"], B, g["Q1"])
        dv = torch.empty((B, C, G0, G1), dtype=torch.float32, device=dev)
        o.gemm(1, 0, C, L, PJ, P["Q1"], C, 0, da1, L, PJ * L, dv, L, C * L, B)
        del da1
        dGx = torch.empty((B * C, G0, 2 * mx), dtype=torch.float32, device=dev)
        dFx = torch.empty_like(dGx)
        dO2 = torch.empty((B, C, 2, K), dtype=torch.float32, device=dev)
        dF2 = torch.empty_like(dO2)
        dpre = dv  # the last layer has no GELU
        for l in reversed(range(self.layers)):
            o.csum(B, C, L, dpre, g[f"b{l + 1}"])
            vin = c["v"][l]
            o.wgrad(C, C, L, dpre, vin, B, g[f"W{l + 1}"])
            dvin = torch.empty_like(dpre)
            o.gemm(1, 0, C, L, C, P[f"W{l + 1}"], C, 0, dpre, L, C * L, dvin, L, C * L, B)
            # spectral path
            o.gemm(0, 1, G0, 2 * mx, G1, dpre, G1, L, AA, G1, 0, dGx, 2 * mx, 2 * G0 * mx, B * C)
            o.gemm(1, 0, 2 * Kp, mx, 2 * G0, Dpiv, 2 * Kp, 0, dGx, mx, 2 * G0 * mx, dO2, mx, 2 * K, B * C)
            o.mix(1, B, C, C, K, dO2, P[f"R{l}"], dF2)
            o.mix(2, B, C, C, K, c["F2"][l], dO2, g[f"R{l}"])
            o.gemm(1, 0, 2 * G0, mx, 2 * Kp, Dpv, 2 * G0, 0, dF2, mx, 2 * K, dFx, mx, 2 * G0 * mx, B * C)
            # dvin += dFx CS^T; below the first layer that is the input's gradient
            # times GELU'(its pre-activation): the previous layer's dpre
            if l > 0:
                o.gemm_ex(0, 1, G0, G1, 2 * mx, dFx, 2 * mx, 2 * G0 * mx, CS, 2 * mx, 0, dvin, G1, L, B * C,
                          beta=1.0, C=dvin, aux=c["pre"][l - 1], act=2)
            else:
                o.gemm(0, 1, G0, G1, 2 * mx, dFx, 2 * mx, 2 * G0 * mx, CS, 2 * mx, 0, dvin, G1, L, B * C, beta=1.0)
            dpre = dvin
        o.csum(B, C, L, dpre, g["b0"])
        o.wgrad(C, NP + 2, L, dpre, c["feats"], B, g["W0"])
        return g

    def adam_step(self, lr, wd=0.0):
        self.step += 1
        for k in self.names:
            self.ops.adam(self.params[k], self.grads[k], self.m[k], self.v[k], lr, self.step, wd=wd)

    def loss_and_grad(self, params, xs, ps, target):
        """Relative-L2 loss per sample (mean) and its gradient w.r.t. the output."""
        out = self.forward(params, xs, ps)
        B = out.shape[0]
        L = out[0].numel()
        dY = torch.empty_like(out)
        loss = torch.empty(B, dtype=torch.float64, device=self.device)
        self.ops.rel_l2(B, L, out, target.contiguous(), dY, loss)
        return float(loss.mean()), dY


# =============================================================================
# Thermal-state data from plain Bloch runs, training, seeded refinement
# =============================================================================
class MorseBlochSetup:
    """The thermal-state workload: Morse V = D (1 - exp(-a (x - x_e)))^2, K = p^2/2,
    on a P x X grid; Bloch exponents exp(-dbeta/4 (V- + V+ - V_min)) and
    exp(-dbeta/2 (K+ + K- - K_min)) as in wigner_bloch_cuda_1d.py:290-359
    (the Gibbs state exp(-beta H))."""

    def __init__(self, grid=512, X_amplitude=8.0, P_amplitude=8.0, x_e=-2.0, dbeta=1e-3):
        self.G, self.XA, self.PA, self.x_e, self.dbeta = int(grid), float(X_amplitude), float(P_amplitude), x_e, dbeta
        G = self.G
        self.dX, self.dP = 2 * self.XA / G, 2 * self.PA / G
        self.X = np.linspace(-self.XA, self.XA - self.dX, G)
        self.P = np.linspace(-self.PA, self.PA - self.dP, G)
        self.Theta = np.fft.fftfreq(G, self.dP / (2 * np.pi))[: G // 2 + 1]
        self.Lambda = np.fft.fftfreq(G, self.dX / (2 * np.pi))[: G // 2 + 1]

    def V(self, D, a):
        x_e = self.x_e
        return lambda x: D * (1.0 - np.exp(-a * (x - x_e))) ** 2

    def tables(self, D, a, dbeta=None):
        db = self.dbeta if dbeta is None else dbeta
        V = self.V(D, a)
        x, th = self.X[None, :], self.Theta[:, None]
        vs = V(x - 0.5 * th) + V(x + 0.5 * th)
        ev = np.exp(-0.25 * db * (vs - vs.min()))
        p, la = self.P[:, None], self.Lambda[None, :]
        ks = 0.5 * (p + 0.5 * la) ** 2 + 0.5 * (p - 0.5 * la) ** 2
        ek = np.exp(-0.5 * db * (ks - ks.min()))
        return ev, ek


class BlochBatch:
    """Plain Bloch propagation of many (D, a) instances on one grid at once
    (per-instance real exponent tables, FP32 states)."""

    def __init__(self, setup: MorseBlochSetup, Ds, As):
        from ._device import ptr
        from ._lib import FW_F32, FW_STEP_FUSED, WignerDesc

        self.s, self.n = setup, len(Ds)
        self.device = require_cuda()
        self.lib = _lib.load()
        G = setup.G
        self.plan = _lib.c_vp()
        check(self.lib.fw_wigner_plan_create(G, G, self.n, FW_F32, ctypes.byref(self.plan)), "fw_wigner_plan_create")
        ev, ek = zip(*[setup.tables(D, a) for D, a in zip(Ds, As)])
        self.tabV = torch.tensor(np.stack(ev), dtype=torch.float32, device=self.device).contiguous()
        self.tabK = torch.tensor(np.stack(ek), dtype=torch.float32, device=self.device).contiguous()
        self.W = torch.empty((self.n, G, G), dtype=torch.float32, device=self.device)
        d = WignerDesc()
        d.w_bstride = G * G
        d.step_kind = FW_STEP_FUSED
        d.tab_bstride = (G // 2 + 1) * G
        d.tab_real = 1
        d.dxdp = setup.dX * setup.dP
        d.in_scale = 1.0
        self._d, self._ptr = d, ptr

    def __del__(self):
        if getattr(self, "plan", None) is not None and self.plan.value:
            self.lib.fw_wigner_plan_destroy(self.plan)
            self.plan = None

    def set_uniform(self):
        self.W.fill_(1.0 / (self.s.dX * self.s.dP * self.s.G * self.s.G))
        return self

    def set_states(self, W):
        self.W.copy_(W)
        s = self.W.sum(dim=(1, 2), dtype=torch.float64) * self.s.dX * self.s.dP
        self.W.div_(s.float()[:, None, None])
        return self

    def run(self, steps):
        if steps <= 0:
            return self
        obs = torch.empty((steps, self.n, 2), dtype=torch.float64, device=self.device)
        d = self._d
        d.W, d.tabV, d.tabK, d.obs_out = self._ptr(self.W), self._ptr(self.tabV), self._ptr(self.tabK), self._ptr(obs)
        check(self.lib.fw_wigner_propagate(self.plan, ctypes.byref(d), int(steps), stream_handle()),
              "fw_wigner_propagate")
        return self


def generate_dataset(setup, n_runs, betas, rng, train_grid=None, chunk_runs=64):
    """Plain Bloch trajectories from W = const for n_runs random (D, a); the
    states at every beta in `betas` (sorted) are recorded, downsampled to
    train_grid^2.  Returns params (N, 3: D, a, beta) and states (N, g, g)."""
    Ds = rng.uniform(2.0, 10.0, size=n_runs)
    As = rng.uniform(0.5, 1.5, size=n_runs)
    betas = np.sort(np.asarray(betas))
    stride = setup.G // (train_grid or setup.G)
    params, states = [], []
    for r0 in range(0, n_runs, chunk_runs):
        Dc, Ac = Ds[r0:r0 + chunk_runs], As[r0:r0 + chunk_runs]
        bb = BlochBatch(setup, Dc, Ac).set_uniform()
        done = 0
        for beta in betas:
            n = int(round(beta / setup.dbeta))
            bb.run(n - done)
            done = n
            snap = bb.W[:, ::stride, ::stride].clone()
            snap /= snap.sum(dim=(1, 2), keepdim=True)
            states.append(snap)
            params.append(np.stack([Dc, Ac, np.full(len(Dc), beta)], axis=1))
        del bb
    P = np.concatenate(params)
    S = torch.cat(states)
    return P, S


def allreduce_mean_(tensors, group=None):
    """Average each tensor over the ranks of `group` in place: one flat buffer,
    one all_reduce (NCCL on GPU tensors, gloo on CPU ones)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if world == 1 or not tensors:
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, group=group)
    flat /= world
    off = 0
    for t in tensors:
        n = t.numel()
        t.view(-1).copy_(flat[off:off + n])
        off += n


def dp_steps_per_epoch(local_n, batch, group=None):
    """Optimizer steps per epoch when every rank trains on its own local_n
    samples: the smallest local_n // batch over the ranks, so that all ranks
    take the same steps (and the same gradient all-reduces)."""
    n = local_n // batch
    if group is None:
        return n
    import torch.distributed as dist

    t = torch.tensor([n], dtype=torch.int64,
                     device="cuda" if dist.get_backend(group) == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return int(t.item())


def normalise_params(P):
    """(D, a, beta) -> network inputs: D/10, a, log(beta)/log(20)."""
    P = np.asarray(P, dtype=np.float64)
    return np.stack([P[:, 0] / 10.0, P[:, 1], np.log(P[:, 2]) / np.log(20.0)], axis=1)


class BlochSurrogate:
    """FNO + the thermal workload: training on plain-Bloch data and seeding."""

    def __init__(self, setup: MorseBlochSetup, net: FNO2d | None = None, train_grid=None, residual=True):
        self.s, self.g = setup, int(train_grid or setup.G)
        self.net = net or FNO2d(n_params=3, width=32, modes=(16, 16), layers=4, proj=128)
        self.xs = (setup.X / setup.XA).astype(np.float32)
        self.ps = (setup.P / setup.PA).astype(np.float32)
        st = setup.G // self.g
        self.xs_t, self.ps_t = self.xs[::st], self.ps[::st]
        self.residual = bool(residual)
        self._xp_full = (torch.tensor(setup.X), torch.tensor(setup.P))
        self._xp_train = (torch.tensor(setup.X[::st]), torch.tensor(setup.P[::st]))

    def baseline(self, P, full=True):
        """Harmonic-approximation Gibbs state of each Morse well (rows of P:
        D, a, beta), the thermal Wigner function of H_h = p^2/2 + w^2 (x-x_e)^2/2
        with w = a sqrt(2 D): exp(-(2/w) tanh(beta w/2) H_h) (hbar = 1), each
        normalised to unit sum on the full or the training grid; (n, g, g) FP32.
        With `residual` the network learns the anharmonic correction to it."""
        P = np.asarray(P, dtype=np.float64)
        x, p = self._xp_full if full else self._xp_train
        x, p = x.to(self.net.device), p.to(self.net.device)
        w = torch.tensor(P[:, 1] * np.sqrt(2.0 * P[:, 0]), device=x.device)
        c = (2.0 / w) * torch.tanh(0.5 * torch.tensor(P[:, 2], device=x.device) * w)
        Hh = 0.5 * p[None, :, None] ** 2 + 0.5 * (w[:, None, None] * (x[None, None, :] - self.s.x_e)) ** 2
        B = torch.exp(-c[:, None, None] * (Hh - Hh.amin(dim=(1, 2), keepdim=True)))
        return (B / B.sum(dim=(1, 2), keepdim=True)).float()

    def train(self, P, S, epochs=20, batch=16, lr=2e-3, rng=None, log=None, group=None):
        """P: (N, 3) raw (D, a, beta); S: (N, g, g) states (normalised to unit sum).

        group: a torch.distributed process group for data-parallel training;
        every rank passes its own samples (P, S) and the same initial
        parameters, and the gradients are averaged over the ranks before each
        Adam step (one all_reduce), so the parameters stay identical."""
        rng = rng or np.random.default_rng(0)
        X = normalise_params(P)
        N = len(X)
        if not self.residual:
            scale = S.abs().amax(dim=(1, 2), keepdim=True)  # per-sample scale: learn the shape
            T = (S / scale).contiguous()
        else:  # the correction to the harmonic baseline, in units of the baseline's peak
            T = torch.empty_like(S)
            for c0 in range(0, N, 512):
                B = self.baseline(P[c0:c0 + 512], full=False)
                T[c0:c0 + 512] = (S[c0:c0 + 512] - B) / B.amax(dim=(1, 2), keepdim=True)
        per_epoch = dp_steps_per_epoch(N, batch, group)
        steps = epochs * per_epoch
        losses = []
        it = 0
        for ep in range(epochs):
            perm = rng.permutation(N)
            for b0 in range(0, per_epoch * batch, batch):
                idx = perm[b0:b0 + batch]
                lr_t = lr * 0.5 * (1 + math.cos(math.pi * it / max(1, steps)))
                loss, dY = self.net.loss_and_grad(X[idx], self.xs_t, self.ps_t, T[torch.as_tensor(idx)])
                self.net.backward(dY)
                if group is not None:
                    allreduce_mean_([self.net.grads[k] for k in self.net.names], group)
                self.net.adam_step(lr_t)
                losses.append(loss)
                it += 1
            if log:
                log(ep, float(np.mean(losses[-max(1, N // batch):])))
        return losses

    def predict(self, Ds, As, beta, chunk=8):
        """Surrogate thermal Wigner functions on the full grid for instances
        (Ds, As) at one beta, each normalised to sum W dXdP = 1; (n, G, G)."""
        Ds, As = np.atleast_1d(Ds), np.atleast_1d(As)
        outs = []
        for c0 in range(0, len(Ds), chunk):
            X = normalise_params(np.stack([Ds[c0:c0 + chunk], As[c0:c0 + chunk],
                                           np.full(len(Ds[c0:c0 + chunk]), beta)], axis=1))
            out = self.net.forward(X, self.xs, self.ps, cache=False)
            if self.residual:
                n = len(Ds[c0:c0 + chunk])
                B = self.baseline(np.stack([Ds[c0:c0 + chunk], As[c0:c0 + chunk], np.full(n, beta)], axis=1))
                out = B + B.amax(dim=(1, 2), keepdim=True) * out
            outs.append(out / (out.double().sum(dim=(1, 2), keepdim=True) * self.s.dX * self.s.dP).float())
        return torch.cat(outs)

    def refine_split(self, beta, refine_fraction=0.2, min_refine=1.0):
        """(beta_s, steps): the surrogate predicts beta_s, the plain Bloch
        refinement runs the remaining steps; beta_s = 0 means no seeding."""
        db = min(beta, max(refine_fraction * beta, min_refine))
        bs = beta - db
        n_total = int(round(beta / self.s.dbeta))
        if bs <= 0:
            return 0.0, n_total
        return bs, n_total - int(round(bs / self.s.dbeta))

    def seeded_gibbs(self, bb: "BlochBatch", Ds, As, beta, refine_fraction=0.2, min_refine=1.0):
        """Gibbs states at `beta` for the instances of `bb` (tables for (Ds, As)):
        surrogate prediction at beta_s, then plain Bloch refinement to beta."""
        bs, n = self.refine_split(beta, refine_fraction, min_refine)
        if bs <= 0:
            bb.set_uniform()
        else:
            bb.set_states(self.predict(Ds, As, bs))
        bb.run(n)
        return bb.W, n

    def plain_gibbs(self, bb: "BlochBatch", beta):
        """The reference path: Bloch steps from W = const (wigner_bloch_cuda_1d.py:129-165)."""
        bb.set_uniform()
        n = int(round(beta / self.s.dbeta))
        bb.run(n)
        return bb.W, n
