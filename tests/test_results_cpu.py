"""Result I/O on the CPU: the Blackman window and the HHG spectrum against
scipy restatements of the reference's post-processing (file_viwer.py:237-260),
and the frame recorder with host tensors."""
import numpy as np
import torch
from scipy import fft as sfft
from scipy.signal import windows

from fastwigner_b200.results import FrameRecorder, blackman, hhg_spectrum


def test_blackman_matches_scipy():
    for n in (1, 2, 3, 10, 101, 1024):
        np.testing.assert_allclose(blackman(n), windows.blackman(n), atol=1e-15)


def test_hhg_spectrum_matches_windowed_fft_and_finds_the_harmonic():
    dt, omega = 0.05, 0.057
    t = np.arange(20000) * dt
    J = np.sin(3 * omega * t) + 1e-3 * np.sin(11 * omega * t)
    om, spec = hhg_spectrum(J, dt, omega)
    ref = np.abs(sfft.fftshift(sfft.fft(windows.blackman(len(J)) * J))) ** 2
    ref /= ref.max()
    np.testing.assert_allclose(spec, ref, rtol=0, atol=1e-13)  # both normalised to a peak of 1
    np.testing.assert_allclose(om, sfft.fftshift(sfft.fftfreq(len(J), dt / (2 * np.pi))) / omega)
    pos = om > 0
    bin_w = 2 * np.pi / (len(J) * dt * omega)  # spacing of the frequency grid in units of omega
    assert abs(om[pos][np.argmax(spec[pos])] - 3.0) <= 0.5 * bin_w
    h11 = spec[pos][np.argmin(abs(om[pos] - 11.0))]
    assert 1e-8 < h11 < 1e-4


def test_frame_recorder_host_tensors(tmp_path):
    rec = FrameRecorder(depth=2)
    W = torch.zeros(4, 3)
    for i in range(5):
        W += 1
        rec.record(t=0.1 * i, wigner=W, prob=torch.arange(3).to(torch.complex64) * i)
    fr = rec.frames()
    assert len(fr) == 5
    for i, f in enumerate(fr):
        assert f["t"] == 0.1 * i
        np.testing.assert_array_equal(f["wigner"], np.full((4, 3), i + 1.0, dtype=np.float32))
        assert f["prob"].dtype == np.complex64
    p = rec.save(tmp_path / "run.npz", dt=0.05, grid=np.array([4, 3]))
    z = np.load(p)
    assert z["settings_dt"] == 0.05
    np.testing.assert_array_equal(z["frame4_wigner"], fr[4]["wigner"])


def test_frame_recorder_take_drains_in_pieces():
    rec = FrameRecorder(depth=2)
    W = torch.zeros(2, 2)
    for i in range(3):
        W += 1
        rec.record(t=i, wigner=W)
    first = rec.take()
    assert [f["t"] for f in first] == [0, 1, 2]
    assert rec.frames() == []
    for i in range(3, 5):
        W += 1
        rec.record(t=i, wigner=W)
    second = rec.take()
    assert [f["t"] for f in second] == [3, 4]
    np.testing.assert_array_equal(second[-1]["wigner"], np.full((2, 2), 5.0, dtype=np.float32))
