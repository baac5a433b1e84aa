"""fw_wigner_propagate_noalloc -- the propagation entry point for callers that
cannot allocate device memory (hosts that hand the library only buffers from
their own fixed device pool, or loops that must not pay cudaMalloc's implicit
device synchronisation between calls).

Checked through the C ABI against fw_wigner_propagate (the plan-based entry
point) on two calls in a row, at the tolerances the other parity tests use
(FP64 1e-10, FP32 1e-5 relative L2), plus the rejection of a batch whose
scratch does not fit the fixed array.  This file is collected last so a run
that stops at the first failure has already run everything else."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = X = 256
BATCH = 3
STEPS = 7


def _setup(dtype_code):
    import torch

    from fastwigner_b200 import _lib

    rt = torch.float64 if dtype_code == _lib.FW_F64 else torch.float32
    ct = torch.complex128 if dtype_code == _lib.FW_F64 else torch.complex64
    dX, dP = 20.0 / X, 20.0 / P
    x = np.linspace(-10, 10 - dX, X)[None, :]
    p = np.linspace(-10, 10 - dP, P)[:, None]
    th = np.fft.fftfreq(P, dP / (2 * np.pi))[: P // 2 + 1][:, None]
    la = np.fft.fftfreq(X, dX / (2 * np.pi))[: X // 2 + 1][None, :]
    V = lambda z: 0.05 * z ** 4 - z ** 2  # noqa: E731
    dt = 0.005
    tabV = torch.view_as_real(torch.tensor(np.exp(-0.5j * dt * (V(x - th / 2) - V(x + th / 2))), dtype=ct,
                                           device="cuda")).contiguous()
    tabK = torch.view_as_real(torch.tensor(np.exp(-1j * dt * ((p + la / 2) ** 2 - (p - la / 2) ** 2) / 2),
                                           dtype=ct, device="cuda")).contiguous()
    rng = np.random.default_rng(7)
    W0 = np.stack([np.exp(-(x - rng.uniform(-2, 2)) ** 2 / 0.25 - 0.25 * (p - rng.uniform(-1, 1)) ** 2)
                   for _ in range(BATCH)])
    W0 /= W0.sum(axis=(1, 2), keepdims=True) * dX * dP
    W = torch.tensor(W0, dtype=rt, device="cuda")
    return W, tabV, tabK, dX * dP


def _desc(W, tabV, tabK, dxdp, obs):
    from fastwigner_b200._lib import FW_STEP_FUSED, WignerDesc

    d = WignerDesc()
    d.W = W.data_ptr()
    d.w_bstride = P * X
    d.step_kind = FW_STEP_FUSED
    d.tabV, d.tabK = tabV.data_ptr(), tabK.data_ptr()
    d.obs_out = obs.data_ptr()
    d.dxdp = dxdp
    d.in_scale = 1.0
    return d


@pytest.mark.parametrize("precision,tol", [("float64", 1e-10), ("float32", 1e-5)])
def test_noalloc_matches_plan_entry_point_on_two_calls(precision, tol):
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    code = _lib.FW_F64 if precision == "float64" else _lib.FW_F32
    W, tabV, tabK, dxdp = _setup(code)
    Wref = W.clone()
    plan = _lib.c_vp()
    _lib.check(lib.fw_wigner_plan_create(P, X, BATCH, code, ctypes.byref(plan)))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        for _ in range(2):
            obs_a = torch.empty((STEPS, BATCH, 2), dtype=torch.float64, device="cuda")
            obs_b = torch.empty_like(obs_a)
            _lib.check(lib.fw_wigner_propagate_noalloc(P, X, BATCH, code, ctypes.byref(_desc(W, tabV, tabK, dxdp,
                                                                                          obs_a)), STEPS, stream))
            _lib.check(lib.fw_wigner_propagate(plan, ctypes.byref(_desc(Wref, tabV, tabK, dxdp, obs_b)), STEPS,
                                               stream))
            torch.cuda.synchronize()
            a, b = W.double().cpu().numpy(), Wref.double().cpu().numpy()
            assert np.isfinite(a).all()
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < tol
            np.testing.assert_allclose(obs_a.cpu().numpy(), obs_b.cpu().numpy(), rtol=tol)
    finally:
        lib.fw_wigner_plan_destroy(plan)


def test_noalloc_rejects_scratch_beyond_its_fixed_size():
    from fastwigner_b200 import _lib

    lib = _lib.load()
    W, tabV, tabK, dxdp = _setup(_lib.FW_F64)
    import torch

    obs = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = lib.fw_wigner_propagate_noalloc(4096, 4096, 60000, _lib.FW_F64, ctypes.byref(_desc(W, tabV, tabK, dxdp, obs)),
                                         1, None)
    assert rc == 1
    assert b"more than the fixed" in lib.fw_last_error()
    assert lib.fw_noalloc_scratch_bytes() == 4 << 20
