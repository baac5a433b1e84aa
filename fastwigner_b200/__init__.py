"""fastwigner_b200: B200-native split-operator propagators for phase-space
quantum dynamics (Moyal, Bloch, von Neumann, random collision, strong field).

The classes are drop-ins for the reference's propagator classes: same
constructor keywords, attributes and methods; the hot path is
libfastwigner.so (sm_100a CUDA) driven through a ctypes C ABI.
"""
from ._lib import FastWignerError
from .wigner import WignerBlochFFTW1D, WignerMoyalFTTW1D, WignerRandomCollisionModelFFTW1D

__all__ = [
    "FastWignerError",
    "WignerMoyalFTTW1D",
    "WignerBlochFFTW1D",
    "WignerRandomCollisionModelFFTW1D",
]

from .rho import RhoBlochCUDA1D, RhoVNeumannCUDA1D
from .strong_field import StrongFieldWigner

__all__ += ["RhoVNeumannCUDA1D", "RhoBlochCUDA1D", "StrongFieldWigner"]

try:  # classes that need the NVRTC expression compiler
    from .wigner_cuda import WignerBlochCUDA1D, WignerMoyalCUDA1D  # noqa: F401

    __all__ += ["WignerMoyalCUDA1D", "WignerBlochCUDA1D"]
except ImportError:  # pragma: no cover - module added incrementally
    pass
