"""Load the reference's own FFTW (CPU) propagators under Python 3.

TEST INFRASTRUCTURE ONLY.  This module is the checker's checker: it lets the
golden-fixture generator (``tests/golden/gen_golden.py``) run the unmodified
reference classes ``WignerMoyalFTTW1D``, ``WignerBlochFFTW1D`` and
``WignerRandomCollisionModelFFTW1D`` in this container, so that the numpy
restatement in ``oracle/wigner_oracle.py`` can be pinned against them.  It is
never imported by the product package, ``bench.py`` or the GPU tests (the
reference tree is not present on GPU hosts).

The reference is Python 2 code written against pyFFTW.  The shim changes
nothing in the reference's arithmetic; it only provides what Python 3 and
this image lack:

* ``xrange`` -> ``range``; ``np.float`` / ``np.complex`` -> builtins;
* 3-argument ``types.MethodType(f, obj, cls)`` (Python 2 bound methods);
* the ``<>`` operator (``wigner_bloch_fftw_1d.py:37``) rewritten to ``!=``
  in the loaded source text;
* a ``pyfftw`` stand-in whose ``FFTW`` plans run ``numpy.fft.rfft`` /
  ``irfft`` along the planned axis, writing into the planned output array
  (the reference aliases its theta-x and p-lambda buffers, so in-place
  semantics matter) with pyFFTW's default ``normalise_idft=True``.

FFT parity is therefore against numpy's pocketfft (FP64), not FFTW: FFTW is
an external library (no version pinned by the reference; call sites
``wigner_moyal_fftw_1d.py:333-366``).
"""
from __future__ import annotations

import builtins
import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

# the reference checkout; FASTWIGNER_REFERENCE overrides the default location
REFERENCE = Path(os.environ.get("FASTWIGNER_REFERENCE", "/root/reference"))


class _FFTWPlan:
    """Stand-in for pyfftw.FFTW: out-of-place r2c / c2r along one axis."""

    def __init__(self, a, b, axes=(0,), direction="FFTW_FORWARD", flags=(), threads=1, **_):
        self.a, self.b = a, b
        self.axis = axes[0]
        self.forward = direction == "FFTW_FORWARD"

    def __call__(self):
        if self.forward:
            self.b[...] = np.fft.rfft(self.a, axis=self.axis)
        else:
            self.b[...] = np.fft.irfft(self.a, n=self.b.shape[self.axis], axis=self.axis)
        return self.b


def _make_pyfftw() -> types.ModuleType:
    m = types.ModuleType("pyfftw")
    m.FFTW = _FFTWPlan
    m.empty_aligned = lambda shape, dtype=float, **_: np.empty(shape, dtype=dtype)
    m.import_wisdom = lambda w: None
    m.export_wisdom = lambda: ()
    return m


def _method_type(f, obj, cls=None):
    return types.MethodType(f, obj)


def _install_globals() -> None:
    builtins.xrange = range
    if not hasattr(np, "float"):
        np.float = float
    if not hasattr(np, "complex"):
        np.complex = complex
    sys.modules.setdefault("pyfftw", _make_pyfftw())


def _load(name: str, ref_root: Path) -> types.ModuleType:
    if name in sys.modules and getattr(sys.modules[name], "__shimmed__", False):
        return sys.modules[name]
    path = ref_root / f"{name}.py"
    src = path.read_text().replace("<>", "!=")
    # the __main__ demos are not executed (module name is not __main__)
    mod = types.ModuleType(name)
    mod.__file__ = str(path)
    mod.__shimmed__ = True
    sys.modules[name] = mod
    code = compile(src, str(path), "exec")
    exec(code, mod.__dict__)
    mod.MethodType = _method_type
    return mod


def load_reference(ref_root: Path = REFERENCE) -> dict:
    """Return the reference FFTW classes, loaded through the shim."""
    _install_globals()
    moyal = _load("wigner_moyal_fftw_1d", ref_root)
    bloch = _load("wigner_bloch_fftw_1d", ref_root)
    coll = _load("wigner_random_collision_model_fftw_1d", ref_root)
    return {
        "WignerMoyalFTTW1D": moyal.WignerMoyalFTTW1D,
        "WignerBlochFFTW1D": bloch.WignerBlochFFTW1D,
        "WignerRandomCollisionModelFFTW1D": coll.WignerRandomCollisionModelFFTW1D,
    }
