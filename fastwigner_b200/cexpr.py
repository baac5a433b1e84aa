"""User C expressions -> NVRTC evaluation modules.

The reference's CUDA classes take C-expression strings (V, K, diff_V,
diff_K, boundaries, initial states, observables) plus ``consts`` and
``functions`` strings, and emit every int/float keyword argument as a
``const int`` / ``const double`` declaration
(wigner_moyal_cuda_1d.py:151-166, rho_vneumann_cuda_1d.py:118-133).
``ExprModule`` reproduces that environment and compiles one evaluation
kernel per expression.  Every kernel sees the variables the reference's
kernels declare -- X, P, X_prime, P_prime, Theta, Lambda, X_minus, X_plus, t,
i, j, indexTotal -- and, when given, the device functions K(P, t) and
V(X, t).  Values are tabulated in FP64; the result may be a double or a
``cuda_complex`` (a pycuda::complex<double>-compatible type).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._device import ptr, stream_handle
from ._lib import FastWignerError, check

SLOTS = ("X", "P", "X_prime", "P_prime", "Theta", "Lambda", "t", "i", "j", "indexTotal")

PRELUDE = r"""
#define _USE_MATH_DEFINES
#ifndef M_PI
#define M_E        2.71828182845904523536
#define M_LOG2E    1.44269504088896340736
#define M_LOG10E   0.434294481903251827651
#define M_LN2      0.693147180559945309417
#define M_LN10     2.30258509299404568402
#define M_PI       3.14159265358979323846
#define M_PI_2     1.57079632679489661923
#define M_PI_4     0.785398163397448309616
#define M_1_PI     0.318309886183790671538
#define M_2_PI     0.636619772367581343076
#define M_2_SQRTPI 1.12837916709551257390
#define M_SQRT2    1.41421356237309504880
#define M_SQRT1_2  0.707106781186547524401
#endif
typedef unsigned long size_t_fw;
// pycuda::complex<double>-compatible value type for user expressions
struct cuda_complex {
  double re, im;
  __device__ cuda_complex() : re(0), im(0) {}
  __device__ cuda_complex(double r) : re(r), im(0) {}
  __device__ cuda_complex(double r, double i) : re(r), im(i) {}
  __device__ double real() const { return re; }
  __device__ double imag() const { return im; }
  __device__ cuda_complex& operator+=(const cuda_complex& o) { re += o.re; im += o.im; return *this; }
  __device__ cuda_complex& operator-=(const cuda_complex& o) { re -= o.re; im -= o.im; return *this; }
  __device__ cuda_complex& operator*=(const cuda_complex& o) {
    double r = re * o.re - im * o.im; im = re * o.im + im * o.re; re = r; return *this; }
  __device__ cuda_complex& operator/=(const cuda_complex& o) {
    double d = o.re * o.re + o.im * o.im; double r = (re * o.re + im * o.im) / d;
    im = (im * o.re - re * o.im) / d; re = r; return *this; }
};
__device__ inline cuda_complex operator+(cuda_complex a, const cuda_complex& b) { return a += b; }
__device__ inline cuda_complex operator-(cuda_complex a, const cuda_complex& b) { return a -= b; }
__device__ inline cuda_complex operator*(cuda_complex a, const cuda_complex& b) { return a *= b; }
__device__ inline cuda_complex operator/(cuda_complex a, const cuda_complex& b) { return a /= b; }
__device__ inline cuda_complex operator+(cuda_complex a, double b) { a.re += b; return a; }
__device__ inline cuda_complex operator+(double b, cuda_complex a) { a.re += b; return a; }
__device__ inline cuda_complex operator-(cuda_complex a, double b) { a.re -= b; return a; }
__device__ inline cuda_complex operator-(double b, const cuda_complex& a) { return cuda_complex(b - a.re, -a.im); }
__device__ inline cuda_complex operator*(cuda_complex a, double b) { a.re *= b; a.im *= b; return a; }
__device__ inline cuda_complex operator*(double b, cuda_complex a) { a.re *= b; a.im *= b; return a; }
__device__ inline cuda_complex operator/(cuda_complex a, double b) { a.re /= b; a.im /= b; return a; }
__device__ inline cuda_complex operator/(double b, const cuda_complex& a) { return cuda_complex(b) / a; }
__device__ inline cuda_complex operator-(const cuda_complex& a) { return cuda_complex(-a.re, -a.im); }
__device__ inline double real(const cuda_complex& a) { return a.re; }
__device__ inline double imag(const cuda_complex& a) { return a.im; }
__device__ inline double real(double a) { return a; }
__device__ inline double imag(double) { return 0.0; }
__device__ inline cuda_complex conj(const cuda_complex& a) { return cuda_complex(a.re, -a.im); }
__device__ inline double norm(const cuda_complex& a) { return a.re * a.re + a.im * a.im; }
__device__ inline double abs(const cuda_complex& a) { return hypot(a.re, a.im); }
__device__ inline double arg(const cuda_complex& a) { return atan2(a.im, a.re); }
__device__ inline cuda_complex exp(const cuda_complex& a) {
  double s, c; sincos(a.im, &s, &c); double e = exp(a.re); return cuda_complex(e * c, e * s); }
__device__ inline cuda_complex log(const cuda_complex& a) { return cuda_complex(log(abs(a)), arg(a)); }
__device__ inline cuda_complex polar(double r, double th) { double s, c; sincos(th, &s, &c); return cuda_complex(r * c, r * s); }
__device__ inline cuda_complex pow(const cuda_complex& a, double p) { return polar(pow(abs(a), p), p * arg(a)); }
__device__ inline cuda_complex sqrt(const cuda_complex& a) { return polar(sqrt(abs(a)), 0.5 * arg(a)); }
"""

KERNEL = r"""
extern "C" __global__ void {name}(const double* __restrict__ in_, long long n_, double* out_re_, double* out_im_)
{{
    const long long k_ = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k_ >= n_) return;
    const double X = in_[k_], P = in_[n_ + k_], X_prime = in_[2 * n_ + k_], P_prime = in_[3 * n_ + k_];
    const double Theta = in_[4 * n_ + k_], Lambda = in_[5 * n_ + k_], t = in_[6 * n_ + k_];
    const size_t i = (size_t)in_[7 * n_ + k_], j = (size_t)in_[8 * n_ + k_];
    const size_t indexTotal = (size_t)in_[9 * n_ + k_];
    const double X_minus = X - 0.5 * Theta, X_plus = X + 0.5 * Theta;
    (void)X; (void)P; (void)X_prime; (void)P_prime; (void)Theta; (void)Lambda; (void)t; (void)i; (void)j;
    (void)indexTotal; (void)X_minus; (void)X_plus;
    const cuda_complex r_ = cuda_complex({expr});
    out_re_[k_] = r_.re;
    if (out_im_) out_im_[k_] = r_.im;
}}
"""

FUNCS = r"""
// Kinetic energy
__device__ double K(double P, double t)
{{
    return ({K});
}}

// Potential energy
__device__ double V(double X, double t)
{{
    return ({V});
}}
"""


def cuda_consts(kwargs: dict, extra: dict | None = None, user_consts: str = "") -> str:
    """const declarations for every int / float keyword, formatted as the
    reference does (wigner_moyal_cuda_1d.py:156-160)."""
    out = ""
    items = dict(kwargs)
    if extra:
        items.update(extra)
    for name, value in items.items():
        if isinstance(value, (bool, np.bool_)):
            out += "    const int %s = %d;\n" % (name, int(value))
        elif isinstance(value, (int, np.integer)):
            out += "    const int %s = %d;\n" % (name, value)
        elif isinstance(value, (float, np.floating)):
            out += "    const double %s = %.15e;\n" % (name, value)
    return out + (user_consts or "")


def module_source(consts: str, functions: str, exprs: dict, K: str | None = None, V: str | None = None) -> str:
    src = PRELUDE + "\n" + consts + "\n" + (functions or "") + "\n"
    if K is not None and V is not None:
        src += FUNCS.format(K=K, V=V)
    for name, e in exprs.items():
        src += KERNEL.format(name=name, expr=e)
    return src


def check_source(src: str) -> None:
    """NVRTC-compile a module without a device (raises FastWignerError with the log)."""
    lib = _lib.load()
    buf = ctypes.create_string_buffer(1 << 16)
    rc = lib.fw_expr_check(src.encode(), buf, len(buf))
    if rc != 0:
        raise FastWignerError(lib.fw_last_error().decode(errors="replace"))


class ExprModule:
    """A compiled set of expression kernels bound to the current device."""

    def __init__(self, consts: str, functions: str, exprs: dict, K: str | None = None, V: str | None = None):
        self.source = module_source(consts, functions, exprs, K, V)
        self.names = list(exprs)
        self._lib = _lib.load()
        self._h = _lib.c_vp()
        rc = self._lib.fw_expr_create(self.source.encode(), ctypes.byref(self._h))
        if rc != 0:
            raise FastWignerError(self._lib.fw_last_error().decode(errors="replace"))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.fw_expr_destroy(h)
            except Exception:
                pass
            self._h = None

    def eval(self, name: str, n: int, complex_out: bool = False, device=None, **coords) -> torch.Tensor:
        """Evaluate kernel `name` at n points; coords maps slot names (SLOTS) to
        arrays/scalars broadcastable to n.  Returns an FP64 (or complex128) tensor."""
        dev = device or torch.device("cuda", torch.cuda.current_device())
        inp = torch.zeros((len(SLOTS), n), dtype=torch.float64, device=dev)
        for key, val in coords.items():
            if key not in SLOTS:
                raise KeyError(key)
            v = val if isinstance(val, torch.Tensor) else torch.from_numpy(np.array(val, dtype=np.float64))
            inp[SLOTS.index(key)] = v.to(dev, torch.float64).reshape(-1).expand(n) if v.numel() == 1 else \
                v.to(dev, torch.float64).reshape(-1)
        re = torch.empty(n, dtype=torch.float64, device=dev)
        im = torch.empty(n, dtype=torch.float64, device=dev) if complex_out else None
        check(self._lib.fw_expr_eval(self._h, name.encode(), ptr(inp), n, ptr(re), ptr(im), stream_handle()),
              f"evaluating {name}")
        return torch.complex(re, im) if complex_out else re

    def eval_grid(self, name: str, shape, complex_out=False, **coords) -> np.ndarray:
        """Evaluate on broadcast numpy coordinate grids; returns a numpy array of `shape`."""
        n = int(np.prod(shape))
        flat = {k: np.broadcast_to(np.asarray(v, dtype=np.float64), shape).reshape(-1) for k, v in coords.items()}
        return self.eval(name, n, complex_out=complex_out, **flat).cpu().numpy().reshape(shape)
