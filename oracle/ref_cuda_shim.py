"""Run the reference's own CUDA-class propagators on the host CPU.

TEST INFRASTRUCTURE ONLY.  Like ``oracle/ref_shim.py`` for the FFTW classes,
this lets the fixture generator (``tests/golden/gen_golden_cuda.py``) run the
UNMODIFIED reference classes ``WignerMoyalCUDA1D``, ``WignerBlochCUDA1D``,
``RhoVNeumannCUDA1D`` and ``RhoBlochCUDA1D`` in this container, so that the
numpy restatements in ``oracle/wigner_oracle.py`` (CUDA convention) and
``oracle/rho_oracle.py`` can be pinned against what those classes compute.
It is never imported by the product package, ``bench.py`` or the GPU tests.

The classes are Python 2 code on PyCUDA, scikit-cuda and a ctypes cuFFT
binding, none of which exists here.  This module is also the build recipe of
their kernels: it supplies stand-ins whose behaviour follows the documented
semantics of each call, and compiles the reference's own kernel sources
(the C strings the classes format and hand to ``SourceModule``) with g++ as
host C++, writing the objects only under ``oracle/_ref/``:

* ``pycuda.gpuarray``: ``GPUArray`` views over host byte buffers standing in
  for device allocations (``gpudata=`` aliasing included: the reference
  shares one allocation between its theta-x and p-lambda spectra), with the
  array arithmetic the classes use; ``sum``, ``dot`` (no conjugation), ``min``,
  ``zeros``, ``empty``, ``empty_like``, ``to_gpu``, ``_memcpy_discontig``.
* ``pycuda.compiler.SourceModule``: the kernel source is compiled with a
  prelude that maps ``pycuda::complex<T>`` to ``std::complex<T>`` and turns
  ``__global__`` / ``__device__`` functions into host functions; a generated
  ``extern "C"`` launcher runs every thread of the launch grid in order
  (the reference's kernels are element-wise: no shared memory, no barriers).
* ``pycuda.reduction.ReductionKernel``: the map expression compiled into a
  sequential FP64 loop.
* ``skcuda.linalg.trace``; ``pycuda.driver.mem_get_info`` (zeros).
* ``cufft`` (the reference's ctypes cuFFT module, cufft.py:105-342): plans
  record their axis; ``cu_fft_D2Z`` / ``cu_ifft_Z2D`` / ``fft_Z2Z`` /
  ``ifft_Z2Z`` run numpy's pocketfft along that axis with cuFFT's
  conventions -- forward unnormalised, inverse unnormalised (no 1/N), a
  complex-to-real inverse keeping only the real part of the DC and Nyquist
  bins.

Python 2 fixes as in ``ref_shim.py`` (xrange, 3-argument MethodType,
``fractions.gcd``, ``np.float``).  FFT parity is against pocketfft, not cuFFT.
"""
from __future__ import annotations

import builtins
import ctypes
import fractions
import hashlib
import math
import os
import re
import subprocess
import sys
import types
from pathlib import Path

import numpy as np

# the reference checkout; FASTWIGNER_REFERENCE overrides the default location
REFERENCE = Path(os.environ.get("FASTWIGNER_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent / "_ref"

# ---------------------------------------------------------------------------
# device memory and arrays


class _Alloc:
    """A device allocation: a zero-filled host byte buffer."""

    def __init__(self, nbytes):
        self.buf = np.zeros(max(int(nbytes), 16), np.uint8)

    def __int__(self):
        return int(self.buf.ctypes.data)


def _val(x):
    return x._a if isinstance(x, GPUArray) else (x.get() if hasattr(x, "get") and not np.isscalar(x) else x)


class GPUArray:
    def __init__(self, shape, dtype=np.float64, gpudata=None, **_):
        shape = tuple(int(s) for s in shape) if np.iterable(shape) else (int(shape),)
        self.shape, self.dtype = shape, np.dtype(dtype)
        n = int(np.prod(shape)) if shape else 1
        self.gpudata = gpudata if gpudata is not None else _Alloc(n * self.dtype.itemsize)
        self._a = np.frombuffer(self.gpudata.buf, self.dtype, count=n).reshape(shape)

    size = property(lambda self: self._a.size)
    nbytes = property(lambda self: self._a.nbytes)
    ndim = property(lambda self: self._a.ndim)

    @classmethod
    def _wrap(cls, arr):
        arr = np.asarray(arr)
        g = cls(arr.shape, arr.dtype)
        g._a[...] = arr
        return g

    def get(self):
        return self._a.copy()

    def set(self, ary):
        self._a[...] = ary

    def fill(self, v):
        self._a.fill(v)
        return self

    def copy(self):
        return GPUArray._wrap(self._a)

    def __setitem__(self, idx, v):
        self._a[idx] = _val(v)

    def __getitem__(self, idx):
        return GPUArray._wrap(self._a[idx])

    def __itruediv__(self, s):
        self._a /= _val(s)
        return self

    def __imul__(self, s):
        self._a *= _val(s)
        return self

    def __iadd__(self, s):
        self._a += _val(s)
        return self

    def __isub__(self, s):
        self._a -= _val(s)
        return self

    def __truediv__(self, s):
        return GPUArray._wrap(self._a / _val(s))

    def __mul__(self, s):
        return GPUArray._wrap(self._a * _val(s))

    __rmul__ = __mul__

    def __add__(self, s):
        return GPUArray._wrap(self._a + _val(s))

    def __sub__(self, s):
        return GPUArray._wrap(self._a - _val(s))

    @property
    def real(self):
        return GPUArray._wrap(self._a.real.copy())

    @property
    def imag(self):
        return GPUArray._wrap(self._a.imag.copy())

    def conj(self):
        return GPUArray._wrap(np.conj(self._a))

    def __len__(self):
        return self.shape[0]


def _make_gpuarray():
    m = types.ModuleType("pycuda.gpuarray")
    m.GPUArray = GPUArray
    m.zeros = lambda shape, dtype=np.float64, **_: GPUArray(shape, dtype)
    m.empty = lambda shape, dtype=np.float64, **_: GPUArray(shape, dtype)
    m.empty_like = lambda a: GPUArray(a.shape, a.dtype)
    m.zeros_like = lambda a: GPUArray(a.shape, a.dtype)
    m.to_gpu = lambda a: GPUArray._wrap(a)
    m.sum = lambda a, **_: GPUArray._wrap(np.sum(a._a))
    m.dot = lambda a, b, **_: GPUArray._wrap(np.sum(a._a * b._a))
    m.min = lambda a, **_: GPUArray._wrap(np.min(a._a))
    m.max = lambda a, **_: GPUArray._wrap(np.max(a._a))

    def memcpy_discontig(dst, src, **_):
        dst._a[...] = src._a

    m._memcpy_discontig = memcpy_discontig
    return m


# ---------------------------------------------------------------------------
# kernels: the reference's C sources compiled as host C++

_PRELUDE = r"""
#include <complex>
#include <cmath>
#include <cstddef>
struct fwref_dim3 { unsigned int x, y, z; };
static fwref_dim3 threadIdx, blockIdx, blockDim, gridDim;
#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline
using std::real; using std::imag; using std::conj; using std::abs; using std::exp; using std::norm;
using std::sqrt; using std::pow; using std::cos; using std::sin; using std::tan; using std::signbit;
"""

_COMPLEX_HPP = r"""
// pycuda::complex<T> of the reference's kernels, as std::complex<T>
#pragma once
#include <complex>
namespace pycuda { template <class T> using complex = std::complex<T>; }
"""

_GLOBAL_RE = re.compile(r"__global__\s+void\s+(\w+)\s*\(([^)]*)\)", re.S)


def _param_types(params: str):
    out = []
    for p in params.split(","):
        p = " ".join(p.split())
        if not p:
            continue
        m = re.match(r"(.*?)(\w+)$", p)
        ty = m.group(1).strip()
        out.append(ty)
    return out


def _ctype_of(ty: str):
    base = ty.replace("const", "").strip()
    if "*" in base:
        return None  # pointer
    return {"double": ctypes.c_double, "float": ctypes.c_float, "int": ctypes.c_int,
            "unsigned int": ctypes.c_uint, "long": ctypes.c_long, "size_t": ctypes.c_size_t}[base]


def _compile(src: str, tag: str) -> ctypes.CDLL:
    OUT.mkdir(parents=True, exist_ok=True)
    inc = OUT / "include"
    inc.mkdir(exist_ok=True)
    hpp = inc / "pycuda-complex.hpp"
    if not hpp.exists():
        hpp.write_text(_COMPLEX_HPP)
    h = hashlib.sha1((tag + src).encode()).hexdigest()[:16]
    so = OUT / f"k_{h}.so"
    if not so.exists():
        cpp = OUT / f"k_{h}.cpp"
        cpp.write_text(src)
        # -ffp-contract=off: no fused multiply-adds the kernel source does not write
        cmd = ["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=c++17", "-shared", "-fPIC",
               "-I", str(inc), str(cpp), "-o", str(so)]
        subprocess.run(cmd, check=True)
    return ctypes.CDLL(str(so))


class _Function:
    def __init__(self, lib, name, types_):
        self._f = getattr(lib, "fwref_launch_" + name)
        self._f.restype = None
        self._f.argtypes = [ctypes.c_int] * 6 + [ctypes.POINTER(ctypes.c_void_p)]
        self._types = types_

    def __call__(self, *args, block=(1, 1, 1), grid=(1, 1), **_):
        if len(args) != len(self._types):
            raise TypeError("kernel argument count mismatch")
        keep = []
        ptrs = (ctypes.c_void_p * max(1, len(args)))()
        for i, (a, ty) in enumerate(zip(args, self._types)):
            ct = _ctype_of(ty)
            if ct is None:
                ptrs[i] = int(a.gpudata) if isinstance(a, GPUArray) else int(a)
            else:
                v = ct(a.item() if hasattr(a, "item") else a)
                keep.append(v)
                ptrs[i] = ctypes.cast(ctypes.byref(v), ctypes.c_void_p)
        g = tuple(grid) + (1,) * (3 - len(grid))
        b = tuple(block) + (1,) * (3 - len(block))
        self._f(int(g[0]), int(g[1]), int(g[2]), int(b[0]), int(b[1]), int(b[2]), ptrs)


class SourceModule:
    """Compile a reference kernel source for the host and expose its kernels."""

    def __init__(self, source, **_):
        kernels = _GLOBAL_RE.findall(source)
        launch = []
        for name, params in kernels:
            tys = _param_types(params)
            args = []
            for i, ty in enumerate(tys):
                if _ctype_of(ty) is None:
                    args.append(f"({ty})a[{i}]")
                else:
                    args.append(f"*({ty.replace('const', '').strip()}*)a[{i}]")
            launch.append(
                f'extern "C" void fwref_launch_{name}(int gx, int gy, int gz, int bx, int by, int bz, void** a) {{\n'
                f"  gridDim = {{(unsigned)gx, (unsigned)gy, (unsigned)gz}};\n"
                f"  blockDim = {{(unsigned)bx, (unsigned)by, (unsigned)bz}};\n"
                f"  for (int z = 0; z < gz; ++z) for (int y = 0; y < gy; ++y) for (int x = 0; x < gx; ++x) {{\n"
                f"    blockIdx = {{(unsigned)x, (unsigned)y, (unsigned)z}};\n"
                f"    for (int tz = 0; tz < bz; ++tz) for (int ty = 0; ty < by; ++ty) for (int tx = 0; tx < bx; ++tx) {{\n"
                f"      threadIdx = {{(unsigned)tx, (unsigned)ty, (unsigned)tz}};\n"
                f"      {name}({', '.join(args)});\n"
                f"    }}\n  }}\n}}\n")
            self._types = getattr(self, "_types", {})
            self._types[name] = tys
        self._lib = _compile(_PRELUDE + source + "\n" + "".join(launch), "module")

    def get_function(self, name):
        return _Function(self._lib, name, self._types[name])


class ReductionKernel:
    """pycuda.reduction.ReductionKernel: map_expr over i, reduced with
    reduce_expr (a, b) from `neutral`, sequentially in the output type."""

    def __init__(self, dtype_out, neutral, reduce_expr, map_expr, arguments, **_):
        self.dtype = np.dtype(dtype_out)
        cty = {np.dtype(np.float64): "double", np.dtype(np.float32): "float"}[self.dtype]
        args = [" ".join(a.split()) for a in arguments.split(",")]
        self._types = [re.match(r"(.*?)(\w+)$", a).group(1).strip() for a in args]
        names = [re.match(r"(.*?)(\w+)$", a).group(2) for a in args]
        unpack = "".join(f"  {t} {n} = ({t})a[{i}];\n" for i, (t, n) in enumerate(zip(self._types, names)))
        src = (_PRELUDE + "#include <pycuda-complex.hpp>\n"
               f'extern "C" {cty} fwref_reduce(long n, void** a) {{\n{unpack}'
               f"  {cty} acc = ({cty})({neutral});\n"
               f"  for (long i = 0; i < n; ++i) {{ {cty} a_ = acc; {cty} b_ = ({map_expr});\n"
               f"    acc = [&]({cty} a, {cty} b) {{ return ({reduce_expr}); }}(a_, b_); }}\n"
               f"  return acc;\n}}\n")
        self._lib = _compile(src, "reduction")
        self._f = self._lib.fwref_reduce
        self._f.restype = {"double": ctypes.c_double, "float": ctypes.c_float}[cty]
        self._f.argtypes = [ctypes.c_long, ctypes.POINTER(ctypes.c_void_p)]

    def __call__(self, *arrays, **_):
        ptrs = (ctypes.c_void_p * len(arrays))(*[int(a.gpudata) for a in arrays])
        return GPUArray._wrap(np.array(self._f(arrays[0].size, ptrs), self.dtype))


def _dtype_to_ctype(dtype):
    dtype = np.dtype(dtype)
    return {np.dtype(np.float64): "double", np.dtype(np.float32): "float",
            np.dtype(np.complex128): "pycuda::complex<double>",
            np.dtype(np.complex64): "pycuda::complex<float>", np.dtype(np.int32): "int"}[dtype]


# ---------------------------------------------------------------------------
# cuFFT stand-in with the reference cufft.py's module interface


def _make_cufft():
    m = types.ModuleType("cufft")
    m.CUFFT_FORWARD, m.CUFFT_INVERSE = -1, 1
    m.CUFFT_R2C, m.CUFFT_C2R, m.CUFFT_C2C = 0x2a, 0x2c, 0x29
    m.CUFFT_D2Z, m.CUFFT_Z2D, m.CUFFT_Z2Z = 0x6a, 0x6c, 0x69

    class _Plan:
        def __init__(self, shape, axes):
            self.shape, self.axes = tuple(shape), axes

    m.Plan2DAxis0 = lambda shape, t=None: _Plan(shape, (0,))
    m.Plan2DAxis1 = lambda shape, t=None: _Plan(shape, (1,))
    m.PlanZ2Z = lambda shape, batch=1: _Plan(shape, tuple(range(len(shape))))
    m.Plan_Z2Z_2D_Axis0 = lambda shape: _Plan(shape, (0,))
    m.Plan_Z2Z_2D_Axis1 = lambda shape: _Plan(shape, (1,))

    def fft_d2z(x, y, plan):
        ax = plan.axes[0]
        y._a[...] = np.fft.rfft(x._a, axis=ax)

    def ifft_z2d(x, y, plan):  # unnormalised complex-to-real
        ax = plan.axes[0]
        n = y._a.shape[ax]
        y._a[...] = np.fft.irfft(x._a, n=n, axis=ax) * n

    def fft_z2z(x, y, plan):
        y._a[...] = np.fft.fftn(x._a, axes=plan.axes)

    def ifft_z2z(x, y, plan):  # unnormalised inverse
        n = int(np.prod([x._a.shape[a] for a in plan.axes]))
        y._a[...] = np.fft.ifftn(x._a, axes=plan.axes) * n

    m.cu_fft_D2Z, m.cu_ifft_Z2D, m.fft_Z2Z, m.ifft_Z2Z = fft_d2z, ifft_z2d, fft_z2z, ifft_z2z
    return m


# ---------------------------------------------------------------------------


def _install() -> None:
    builtins.xrange = range
    if not hasattr(np, "float"):
        np.float = float
    if not hasattr(np, "complex"):
        np.complex = complex
    fractions.gcd = math.gcd
    pycuda = types.ModuleType("pycuda")
    ga = _make_gpuarray()
    comp = types.ModuleType("pycuda.compiler")
    comp.SourceModule = SourceModule
    tools = types.ModuleType("pycuda.tools")
    tools.dtype_to_ctype = _dtype_to_ctype
    red = types.ModuleType("pycuda.reduction")
    red.ReductionKernel = ReductionKernel
    drv = types.ModuleType("pycuda.driver")
    drv.mem_get_info = lambda: (0, 0)
    auto = types.ModuleType("pycuda.autoinit")
    pycuda.gpuarray, pycuda.compiler, pycuda.tools = ga, comp, tools
    pycuda.reduction, pycuda.driver, pycuda.autoinit = red, drv, auto
    for name, mod in [("pycuda", pycuda), ("pycuda.gpuarray", ga), ("pycuda.compiler", comp),
                      ("pycuda.tools", tools), ("pycuda.reduction", red), ("pycuda.driver", drv),
                      ("pycuda.autoinit", auto)]:
        sys.modules[name] = mod
    skcuda = types.ModuleType("skcuda")
    lin = types.ModuleType("skcuda.linalg")
    lin.init = lambda: None
    lin.trace = lambda a, **_: np.trace(a._a)
    skcuda.linalg = lin
    sys.modules["skcuda"], sys.modules["skcuda.linalg"] = skcuda, lin
    sys.modules["cufft"] = _make_cufft()


def _method_type(f, obj, cls=None):
    return types.MethodType(f, obj)


def _load(name: str, ref_root: Path) -> types.ModuleType:
    key = "fwref_cuda_" + name
    if key in sys.modules:
        return sys.modules[key]
    path = ref_root / f"{name}.py"
    src = path.read_text().replace("<>", "!=")
    mod = types.ModuleType(name)
    mod.__file__ = str(path)
    sys.modules[key] = mod
    sys.modules[name] = mod  # the Bloch modules import their parent class by module name
    exec(compile(src, str(path), "exec"), mod.__dict__)
    mod.MethodType = _method_type
    mod.pycuda = sys.modules["pycuda"]
    return mod


def load_reference_cuda(ref_root: Path = REFERENCE) -> dict:
    """Return the reference CUDA classes, loaded through the host stand-ins."""
    _install()
    mods = {n: _load(n, ref_root) for n in ("wigner_moyal_cuda_1d", "wigner_bloch_cuda_1d",
                                             "rho_vneumann_cuda_1d", "rho_bloch_cuda_1d")}
    return {
        "WignerMoyalCUDA1D": mods["wigner_moyal_cuda_1d"].WignerMoyalCUDA1D,
        "WignerBlochCUDA1D": mods["wigner_bloch_cuda_1d"].WignerBlochCUDA1D,
        "RhoVNeumannCUDA1D": mods["rho_vneumann_cuda_1d"].RhoVNeumannCUDA1D,
        "RhoBlochCUDA1D": mods["rho_bloch_cuda_1d"].RhoBlochCUDA1D,
    }
