"""Frame recorder with device tensors: each frame holds the state at the
moment it was recorded although the caller keeps updating the tensor on the
same stream right away, including when the ring of slots wraps."""
import numpy as np
import pytest
import torch

from fastwigner_b200.results import FrameRecorder

pytestmark = pytest.mark.gpu


def test_frames_are_snapshots_in_stream_order(tmp_path):
    W = torch.zeros((512, 512), dtype=torch.float32, device="cuda")
    rho_diag = torch.zeros(512, dtype=torch.complex64, device="cuda")
    rec = FrameRecorder(depth=3)
    for i in range(10):
        W.add_(1.0)
        rho_diag.add_(1j)
        rec.record(t=0.5 * i, wigner=W, prob=rho_diag)
        W.mul_(0.0).add_(-7.0)  # overwrite at once; the frame must keep i + 1
        W.fill_(float(i + 1))
    frames = rec.frames()
    assert [f["t"] for f in frames] == [0.5 * i for i in range(10)]
    for i, f in enumerate(frames):
        assert f["wigner"].dtype == np.float32 and f["prob"].dtype == np.complex64
        np.testing.assert_array_equal(f["wigner"], np.full((512, 512), i + 1.0, dtype=np.float32))
        np.testing.assert_array_equal(f["prob"], np.full(512, 1j * (i + 1), dtype=np.complex64))
    z = np.load(rec.save(tmp_path / "frames.npz", X_amplitude=10.0))
    np.testing.assert_array_equal(z["frame9_wigner"], frames[9]["wigner"])


@pytest.mark.parametrize("gamma", [None, 3e-3])
def test_propagate_with_frames_equals_chunked_calls(gamma):
    """propagate(steps, frames=rec, frame_every=k) -- no wait between frames,
    Ehrenfest lists filled at the end -- gives the same frames, final state and
    Ehrenfest lists as a loop of propagate(k) + record (strong field, velocity
    gauge, field integrated from E, with and without collisions)."""
    from fastwigner_b200.strong_field import StrongFieldWigner

    def make():
        kw = dict(X_gridDIM=256, X_amplitude=40.0, P_gridDIM=128, P_amplitude=4.0, dt=0.05, t=0.0,
                  V=lambda _, x: -1.0 / np.sqrt(x * x + 1.0), diff_V=lambda _, x: x / (x * x + 1.0) ** 1.5,
                  gauge="velocity", E=lambda _, t: 0.05 * np.sin(0.057 * t), precision="float64")
        if gamma is not None:
            kw.update(gamma=gamma, kT=0.2, dbeta=0.01)
        q = StrongFieldWigner(**kw)
        q.set_wignerfunction(lambda _, x, p: np.exp(-(x - 1.0) ** 2 - p ** 2) + 0 * x * p)
        return q

    a, b = make(), make()
    ra, rb = FrameRecorder(depth=2), FrameRecorder(depth=2)
    Wa = a.propagate(35, frames=ra, frame_every=10)
    for n in (10, 10, 10, 5):
        b.propagate(n)
        if n == 10:
            rb.record(t=b.t, wigner=b.wigner_device)
    Wb = b.wignerfunction
    np.testing.assert_allclose(Wa, Wb, rtol=0, atol=1e-14)
    fa, fb = ra.frames(), rb.frames()
    assert [f["t"] for f in fa] == [f["t"] for f in fb] and len(fa) == 3
    for x, y in zip(fa, fb):
        np.testing.assert_allclose(x["wigner"], y["wigner"], rtol=0, atol=1e-14)
    for k in ("X_average", "P_average", "X_average_RHS", "P_average_RHS", "hamiltonian_average"):
        np.testing.assert_allclose(getattr(a, k), getattr(b, k), rtol=1e-13, atol=1e-15)
    assert abs(a.t - b.t) < 1e-12
