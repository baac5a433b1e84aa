"""The FNO's batched GEMM on the tensor cores (tcgen05, TF32 three-way split)
against an FP64 numpy product: both tensor-core orientations (N >= M: the
tensor core's rows run along C's contiguous dimension; N < M), every
transpose, the 16/32/64/128-wide column tiles, ragged edges (sizes that are
not multiples of the tiles, K not a multiple of the 32-wide K chunk), alpha
and beta, batches, and the shapes the surrogate uses.  Tolerance 1e-5 of the
largest |C| (FP32 accuracy with FP32 accumulation over K up to 4096; measured
~2e-6 at K = 200; a plain TF32 product is ~1e-3 off).  The status word stays
0."""
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
                                   (512, 16, 512), (128, 128, 96)])
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
