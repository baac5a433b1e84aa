"""Result I/O for long propagations: an asynchronous device-to-host frame
ring written to ``.npz``, and the high-harmonic spectrum of <p>(t).

The reference records every N-th state of a strong-field run into an HDF5
file, one group per frame holding the Wigner function, the time and the
diagonal of rho (strong_field_physics_cuda_1d.py:110-122, 217-249), and
post-processes the dipole velocity <p>(t) into an HHG spectrum
(file_viwer.py:237-260).  Here frames are copied from the device into a ring
of pinned host buffers on a side stream, so that recording a frame does not
wait for the copy, and the collected frames are written as one ``.npz``
archive (h5py is not a dependency of this package).
"""
from __future__ import annotations

import numpy as np
import torch


def blackman(n: int) -> np.ndarray:
    """Symmetric Blackman window of n points:
    0.42 - 0.5 cos(2 pi k/(n-1)) + 0.08 cos(4 pi k/(n-1))."""
    if n < 1:
        return np.zeros(0)
    if n == 1:
        return np.ones(1)
    k = np.arange(n)
    x = 2.0 * np.pi * k / (n - 1)
    return 0.42 - 0.5 * np.cos(x) + 0.08 * np.cos(2.0 * x)


def hhg_spectrum(P_average, dt: float, omega: float):
    """High-harmonic spectrum from the dipole velocity <p>(t) sampled every dt
    (file_viwer.py:237-260): the Blackman-windowed FFT, |.|^2 in centred
    frequency order normalised to a maximum of 1, against frequency in units
    of the laser frequency omega.  Returns (omegas / omega, spectrum)."""
    J = np.asarray(P_average, dtype=np.float64)
    N = len(J)
    F = np.fft.fft(blackman(N) * J)
    spectrum = np.abs(np.fft.fftshift(F)) ** 2
    spectrum /= spectrum.max()
    omegas = np.fft.fftshift(np.fft.fftfreq(N, dt / (2.0 * np.pi))) / omega
    return omegas, spectrum


class FrameRecorder:
    """Asynchronous device -> host recorder of frames (dicts of tensors plus
    scalars).

    ``record(t=..., wigner=tensor, prob=tensor)`` snapshots the device tensors
    into the next slot of a ring of ``depth`` device buffers on the caller's
    stream (an HBM copy, ordered with the propagation, so the caller may go on
    updating the tensors at once), then copies the snapshot into pinned host
    buffers of its own (torch's caching host allocator) on a side stream and
    returns without waiting; the frames hand those buffers out as numpy arrays.  When
    the ring wraps, the oldest slot's copy is waited for and the frame moved
    to the frame list.  ``frames()`` drains the ring; ``save(path,
    **settings)`` writes one ``.npz``: ``settings_<key>`` entries and
    ``frame<i>_<name>`` entries per frame."""

    def __init__(self, depth: int = 4):
        self.depth = max(1, int(depth))
        self._slots = []
        self._next = 0
        self._done = []
        self._count = 0
        self._stream = None

    def _retire(self, slot):
        if slot.get("event") is None:
            return
        slot["event"].synchronize()
        # each frame owns its pinned buffers (from torch's caching host
        # allocator): hand them out as numpy views, no host copy
        frame = {k: v.numpy() for k, v in slot["host"].items()}
        frame.update(slot["scalars"])
        self._done.append((slot["index"], frame))
        slot["event"] = None
        slot["host"] = {}

    @staticmethod
    def _fit(store, k, v, **kw):
        if k not in store or store[k].shape != v.shape or store[k].dtype != v.dtype:
            store[k] = torch.empty(v.shape, dtype=v.dtype, **kw)
        return store[k]

    def record(self, **items):
        """Enqueue one frame; tensors keep their dtype (complex included),
        other items are stored as given."""
        tensors = {k: v.detach() for k, v in items.items() if isinstance(v, torch.Tensor)}
        scalars = {k: v for k, v in items.items() if not isinstance(v, torch.Tensor)}
        if len(self._slots) < self.depth:
            self._slots.append({"host": {}, "dev": {}, "event": None})
        slot = self._slots[self._next]
        self._retire(slot)  # the ring wrapped: finish this slot's previous frame first
        host, dev = slot["host"], slot["dev"]
        for store in (host, dev):
            for k in [k for k in store if k not in tensors]:
                del store[k]
        on_gpu = any(v.is_cuda for v in tensors.values())
        if on_gpu:
            if self._stream is None:
                self._stream = torch.cuda.Stream()
            for k, v in tensors.items():  # snapshot on the caller's stream
                self._fit(dev, k, v, device=v.device).copy_(v)
            self._stream.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(self._stream):
                for k, v in tensors.items():
                    host[k] = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                    host[k].copy_(dev[k], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self._stream)
            slot.update(event=ev, scalars=scalars, index=self._count)
        else:
            frame = {k: v.numpy().copy() for k, v in tensors.items()}
            frame.update(scalars)
            self._done.append((self._count, frame))
        self._count += 1
        self._next = (self._next + 1) % self.depth

    def frames(self):
        """All recorded frames in order (waits for the copies still in flight)."""
        for slot in self._slots:
            self._retire(slot)
        self._done.sort(key=lambda f: f[0])
        return [f for _, f in self._done]

    def take(self):
        """frames(), after which the recorder forgets them (its buffers stay
        allocated for the next frames): for long runs drained in pieces."""
        out = self.frames()
        self._done = []
        return out

    def save(self, path, **settings):
        out = {f"settings_{k}": np.asarray(v) for k, v in settings.items()}
        for i, frame in enumerate(self.frames()):
            for k, v in frame.items():
                out[f"frame{i}_{k}"] = np.asarray(v)
        np.savez(path, **out)
        return path
