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
