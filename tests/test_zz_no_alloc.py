"""fw_wigner_propagate_noalloc -- the propagation entry point for callers that
cannot allocate device memory (hosts that hand the library only buffers from
their own fixed device pool, or loops that must not pay cudaMalloc's implicit
device synchronisation between calls).

Checked through the C ABI against fw_wigner_propagate (the plan-based entry
point) on two calls in a row, at the tolerances the other parity tests use
(FP64 1e-10, FP32 1e-5 relative L2), over: a small batch (small-batch launch
shapes, every CTA reducing the partial sums), a large one on a non-square
grid (regular shapes, per-instance totals kernel, the other row-pass stage
table), with and without x- and p-observables (the fused mid-point column pass
with its weight spectra in the fixed array); a sequence of calls of different
sizes (the twiddles are rewritten on every call); the scratch-size query; and
the rejection of a batch whose scratch does not fit.  This file is collected
last so a run that stops at the first failure has already run everything
else."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 7


def _V(z):
    return 0.05 * z ** 4 - z ** 2


def _setup(P, X, batch, dtype_code, seed=7):
    import torch

    from fastwigner_b200 import _lib

    rt = torch.float64 if dtype_code == _lib.FW_F64 else torch.float32
    ct = torch.complex128 if dtype_code == _lib.FW_F64 else torch.complex64
    dX, dP = 20.0 / X, 20.0 / P
    x = np.linspace(-10, 10 - dX, X)[None, :]
    p = np.linspace(-10, 10 - dP, P)[:, None]
    th = np.fft.fftfreq(P, dP / (2 * np.pi))[: P // 2 + 1][:, None]
    la = np.fft.fftfreq(X, dX / (2 * np.pi))[: X // 2 + 1][None, :]
    dt = 0.005
    tabV = torch.view_as_real(torch.tensor(np.exp(-0.5j * dt * (_V(x - th / 2) - _V(x + th / 2))), dtype=ct,
                                           device="cuda")).contiguous()
    tabK = torch.view_as_real(torch.tensor(np.exp(-1j * dt * ((p + la / 2) ** 2 - (p - la / 2) ** 2) / 2),
                                           dtype=ct, device="cuda")).contiguous()
    rng = np.random.default_rng(seed)
    W0 = np.stack([np.exp(-(x - rng.uniform(-2, 2)) ** 2 / 0.25 - 0.25 * (p - rng.uniform(-1, 1)) ** 2)
                   for _ in range(batch)])
    W0 /= W0.sum(axis=(1, 2), keepdims=True) * dX * dP
    W = torch.tensor(W0, dtype=rt, device="cuda")
    wx = torch.tensor(np.stack([x[0], 0.2 * x[0] ** 3 - 2 * x[0], _V(x[0])]), dtype=torch.float64, device="cuda")
    wp = torch.tensor(np.stack([p[:, 0], p[:, 0], 0.5 * p[:, 0] ** 2]), dtype=torch.float64, device="cuda")
    return dict(P=P, X=X, batch=batch, W=W, tabV=tabV, tabK=tabK, dxdp=dX * dP, wx=wx, wp=wp)


def _desc(c, W, obs, observables):
    from fastwigner_b200._lib import FW_STEP_FUSED, WignerDesc

    d = WignerDesc()
    d.W = W.data_ptr()
    d.w_bstride = c["P"] * c["X"]
    d.step_kind = FW_STEP_FUSED
    d.tabV, d.tabK = c["tabV"].data_ptr(), c["tabK"].data_ptr()
    if observables:
        d.Mx = d.Mp = 3
        d.wx, d.wp = c["wx"].data_ptr(), c["wp"].data_ptr()
    d.obs_out = obs.data_ptr()
    d.dxdp = c["dxdp"]
    d.in_scale = 1.0
    return d


def _compare_one_call(lib, code, c, plan, W, Wref, observables, tol, stream):
    import torch

    from fastwigner_b200 import _lib

    M = 8 if observables else 2
    obs_a = torch.empty((STEPS, c["batch"], M), dtype=torch.float64, device="cuda")
    obs_b = torch.empty_like(obs_a)
    _lib.check(lib.fw_wigner_propagate_noalloc(c["P"], c["X"], c["batch"], code,
                                               ctypes.byref(_desc(c, W, obs_a, observables)), STEPS, stream))
    _lib.check(lib.fw_wigner_propagate(plan, ctypes.byref(_desc(c, Wref, obs_b, observables)), STEPS, stream))
    torch.cuda.synchronize()
    a, b = W.double().cpu().numpy(), Wref.double().cpu().numpy()
    assert np.isfinite(a).all()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < tol
    np.testing.assert_allclose(obs_a.cpu().numpy(), obs_b.cpu().numpy(), rtol=tol, atol=tol * 1e-3)


def _plan(lib, c, code):
    from fastwigner_b200 import _lib

    plan = _lib.c_vp()
    _lib.check(lib.fw_wigner_plan_create(c["P"], c["X"], c["batch"], code, ctypes.byref(plan)))
    return plan


@pytest.mark.parametrize("P,X,batch", [(256, 256, 3), (256, 512, 64)])
@pytest.mark.parametrize("observables", [False, True])
@pytest.mark.parametrize("precision,tol", [("float64", 1e-10), ("float32", 1e-5)])
def test_noalloc_matches_plan_entry_point_on_two_calls(P, X, batch, observables, precision, tol):
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    code = _lib.FW_F64 if precision == "float64" else _lib.FW_F32
    c = _setup(P, X, batch, code)
    W, Wref = c["W"], c["W"].clone()
    plan = _plan(lib, c, code)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        for _ in range(2):
            _compare_one_call(lib, code, c, plan, W, Wref, observables, tol, stream)
    finally:
        lib.fw_wigner_plan_destroy(plan)


def test_noalloc_calls_of_changing_sizes():
    """One size, another size, the first size again: every call rebuilds the
    twiddle tables it needs in the shared array."""
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    code = _lib.FW_F64
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [_setup(256, 256, 3, code, seed=1), _setup(512, 128, 8, code, seed=2)]
    plans = [_plan(lib, c, code) for c in cases]
    refs = [c["W"].clone() for c in cases]
    try:
        for i in (0, 1, 0):
            _compare_one_call(lib, code, cases[i], plans[i], cases[i]["W"], refs[i], True, 1e-10, stream)
    finally:
        for p in plans:
            lib.fw_wigner_plan_destroy(p)


def test_noalloc_scratch_query_and_rejection():
    import torch

    from fastwigner_b200 import _lib

    lib = _lib.load()
    c = _setup(256, 256, 3, _lib.FW_F64)
    obs = torch.empty(1, dtype=torch.float64, device="cuda")
    d = _desc(c, c["W"], obs, True)
    fixed = lib.fw_noalloc_scratch_bytes()
    assert fixed == 4 << 20
    need = lib.fw_noalloc_scratch_needed(256, 256, 3, _lib.FW_F64, ctypes.byref(d))
    assert 0 < need <= fixed
    assert lib.fw_noalloc_scratch_needed(256, 256, 3, _lib.FW_F64, None) < need  # no weight spectra
    assert lib.fw_noalloc_scratch_needed(101, 256, 3, _lib.FW_F64, None) == 0  # odd: rejected
    big = lib.fw_noalloc_scratch_needed(4096, 4096, 60000, _lib.FW_F64, ctypes.byref(d))
    assert big > fixed
    rc = lib.fw_wigner_propagate_noalloc(4096, 4096, 60000, _lib.FW_F64, ctypes.byref(d), 1, None)
    assert rc == 1
    assert b"more than the fixed" in lib.fw_last_error()
