"""The FNO's batched GEMM on the tensor cores (tcgen05, TF32 three-way split)
against an FP64 numpy product: both tensor-core orientations (N >= M: the
tensor core's rows run along C's contiguous dimension; N < M), every
transpose, the 16/32/64/128-wide column tiles, ragged edges (sizes that are
not multiples of the tiles, K not a multiple of the 32-wide K chunk, rows not
16-byte aligned so the float4 loads are off), alpha and beta, batches, the
shapes the surrogate uses, the fused epilogues (bias, pre-activation, GELU,
GELU'), the split-K weight gradient and the fused projection.  Tolerance 1e-5
of the largest |C| (FP32 accuracy with FP32 accumulation over K up to 4096;
measured ~2e-6 at K = 200; a plain TF32 product is ~1e-3 off).  The status
word stays 0."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(ta, tb, M, N, K, alpha, beta, batch, rng):
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    A = rng.normal(size=(batch, K, M) if ta else (batch, M, K))
    B = rng.normal(size=(batch, N, K) if tb else (batch, K, N))
    C0 = rng.normal(size=(batch, M, N))
    At = torch.tensor(A, dtype=torch.float32, device="cuda")
    Bt = torch.tensor(B, dtype=torch.float32, device="cuda")
    Ct = torch.tensor(C0, dtype=torch.float32, device="cuda")
    lda, ldb = (M if ta else K), (K if tb else N)
    _lib.check(lib.fw_fno_sgemm(ta, tb, M, N, K, alpha, ctypes.c_void_p(At.data_ptr()), lda, At[0].numel(),
                                ctypes.c_void_p(Bt.data_ptr()), ldb, Bt[0].numel(), beta,
                                ctypes.c_void_p(Ct.data_ptr()), N, M * N, batch, None))
    torch.cuda.synchronize()
    A32 = At.double().cpu().numpy()
    B32 = Bt.double().cpu().numpy()
    opA = np.transpose(A32, (0, 2, 1)) if ta else A32
    opB = np.transpose(B32, (0, 2, 1)) if tb else B32
    ref = alpha * opA @ opB + beta * C0.astype(np.float32).astype(np.float64)
    return Ct.double().cpu().numpy(), ref


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
@pytest.mark.parametrize("M,N,K", [(32, 300, 32), (130, 16, 200), (64, 64, 8), (200, 100, 45), (16, 1000, 33),
                                   (512, 16, 512), (128, 128, 96), (5, 7, 3), (1, 333, 130), (40, 3, 1)])
def test_tensor_core_gemm_matches_fp64(ta, tb, M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K + 11 * ta + 5 * tb)
    got, ref = _gemm(ta, tb, M, N, K, 1.3, 0.7, 3, rng)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


def test_surrogate_shapes_and_status():
    """The channel map (32 x L x 32), the projection (128 x L x 32) and a
    truncated DFT (512 x 16 x 512, 64-fold batch) of the 512^2 surrogate."""
    from fastwigner_b200 import _lib

    rng = np.random.default_rng(5)
    for (ta, tb, M, N, K, batch) in [(0, 0, 32, 4096, 32, 2), (0, 0, 128, 4096, 32, 2), (0, 0, 512, 16, 512, 4),
                                     (1, 0, 32, 4096, 32, 2), (0, 1, 32, 32, 4096, 2)]:
        got, ref = _gemm(ta, tb, M, N, K, 1.0, 0.0, batch, rng)
        assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-5, (ta, tb, M, N, K)
    st = ctypes.c_int(-1)
    _lib.check(_lib.load().fw_fno_status(ctypes.byref(st), 1))
    assert st.value == 0


def _t(a):
    import torch

    return torch.tensor(a, dtype=torch.float32, device="cuda")


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _gelu(x):
    from scipy.special import erf

    return 0.5 * x * (1 + erf(x / np.sqrt(2)))


def _gelu_d(x):
    from scipy.special import erf

    return 0.5 * (1 + erf(x / np.sqrt(2))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


@pytest.mark.parametrize("act", [0, 1, 2])
@pytest.mark.parametrize("M,N,K", [(32, 4096, 32), (128, 200, 40), (300, 20, 17)])
def test_fused_epilogue(act, M, N, K):
    """out = act(alpha A B + beta C + bias[m]) with pre stored; act 2 multiplies
    by GELU'(aux)."""
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(M + N + K + act)
    batch = 2
    A, B, C0 = rng.normal(size=(batch, M, K)), rng.normal(size=(batch, K, N)), rng.normal(size=(batch, M, N))
    bias, aux = rng.normal(size=M), rng.normal(size=(batch, M, N))
    At, Bt, Ct, bt, xt = _t(A), _t(B), _t(C0), _t(bias), _t(aux)
    pre = torch.empty_like(Ct)
    out = torch.empty_like(Ct)
    _lib.check(lib.fw_fno_sgemm_ex(0, 0, M, N, K, 0.9, _p(At), K, M * K, _p(Bt), N, K * N, 0.5, _p(Ct), N, M * N,
                                   batch, _p(bt), _p(pre), _p(xt), act, _p(out), None))
    torch.cuda.synchronize()
    f = lambda t: t.double().cpu().numpy()
    t = 0.9 * f(At) @ f(Bt) + 0.5 * f(Ct) + f(bt)[None, :, None]
    ref = t if act == 0 else (_gelu(t) if act == 1 else t * _gelu_d(f(xt)))
    assert np.abs(f(pre) - t).max() / np.abs(t).max() < 1e-5
    assert np.abs(f(out) - ref).max() / np.abs(ref).max() < 1e-5


def test_gelu_pointwise_accuracy():
    """The epilogue's GELU and GELU' against the exact functions on a dense
    grid of FP32 arguments in [-12, 12]: within 3e-7 max(1, |x|) (FP32 rounding
    of the result alone is 0.6e-7 |x|).  The GEMM term is zero (K = 1, zero
    operands), so out = act(C)."""
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    M, N = 512, 1024
    x = np.linspace(-12.0, 12.0, M * N).astype(np.float32).reshape(1, M, N)
    xt, ones = _t(x), _t(np.ones_like(x))
    zA, zB = _t(np.zeros((1, M, 1))), _t(np.zeros((1, 1, N)))
    xd = x.astype(np.float64)
    for act, cin, aux, ref in ((1, xt, None, _gelu(xd)), (2, ones, xt, _gelu_d(xd))):
        out = torch.empty_like(xt)
        _lib.check(lib.fw_fno_sgemm_ex(0, 0, M, N, 1, 1.0, _p(zA), 1, M, _p(zB), N, N, 1.0, _p(cin), N, M * N, 1,
                                       None, None, _p(aux) if aux is not None else None, act, _p(out), None))
        torch.cuda.synchronize()
        err = np.abs(out.double().cpu().numpy() - ref) / np.maximum(1.0, np.abs(xd))
        assert err.max() < 3e-7, (act, err.max())


@pytest.mark.parametrize("rows,cols,L,batch", [(32, 32, 65536, 16), (128, 32, 4096, 3), (1, 128, 10000, 4),
                                               (32, 5, 1000, 2), (7, 3, 37, 5)])
def test_split_k_weight_gradient(rows, cols, L, batch):
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(rows * cols + L)
    dY, X = rng.normal(size=(batch, rows, L)), rng.normal(size=(batch, cols, L))
    dYt, Xt = _t(dY), _t(X)
    n = ctypes.c_longlong(0)
    _lib.check(lib.fw_fno_wgrad_work(rows, cols, L, batch, ctypes.byref(n)))
    assert n.value >= batch * rows * cols
    work = torch.empty(n.value, dtype=torch.float32, device="cuda")
    out = torch.full((rows, cols), 0.25, dtype=torch.float32, device="cuda")
    _lib.check(lib.fw_fno_wgrad(rows, cols, L, _p(dYt), rows * L, _p(Xt), cols * L, batch, _p(work), n.value,
                                _p(out), 1, None))
    torch.cuda.synchronize()
    ref = 0.25 + np.einsum("brl,bcl->rc", dYt.double().cpu().numpy(), Xt.double().cpu().numpy())
    assert np.abs(out.double().cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-5
    assert lib.fw_fno_wgrad(rows, cols, L, _p(dYt), rows * L, _p(Xt), cols * L, batch, _p(work), n.value - 1,
                            _p(out), 1, None) != 0


@pytest.mark.parametrize("hidden,C,L", [(128, 32, 5000), (100, 32, 4096), (64, 8, 300)])
def test_fused_projection(hidden, C, L):
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(hidden + C + L)
    batch = 3
    V, Q1, c1 = rng.normal(size=(batch, C, L)), rng.normal(size=(hidden, C)) / np.sqrt(C), rng.normal(size=hidden)
    Q2, c2 = rng.normal(size=hidden) / np.sqrt(hidden), rng.normal(size=1)
    Vt, Q1t, c1t, Q2t, c2t = _t(V), _t(Q1), _t(c1), _t(Q2), _t(c2)
    out = torch.empty((batch, L), dtype=torch.float32, device="cuda")
    _lib.check(lib.fw_fno_project(hidden, C, L, _p(Vt), C * L, batch, _p(Q1t), _p(c1t), _p(Q2t), _p(c2t), _p(out), L,
                                  None))
    torch.cuda.synchronize()
    f = lambda t: t.double().cpu().numpy()
    h = np.einsum("jc,bcl->bjl", f(Q1t), f(Vt)) + f(c1t)[None, :, None]
    ref = f(c2t)[0] + np.einsum("j,bjl->bl", f(Q2t), _gelu(h))
    assert np.abs(f(out) - ref).max() / np.abs(ref).max() < 1e-5
    st = ctypes.c_int(-1)
    _lib.check(lib.fw_fno_status(ctypes.byref(st), 1))
    assert st.value == 0
