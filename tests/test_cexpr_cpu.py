"""NVRTC compilation of reference-style C expressions (runs without a GPU)."""
import pytest

from fastwigner_b200 import cexpr
from fastwigner_b200._lib import FastWignerError

# the strong-field script's strings (strong_field_physics_cuda_1d.py:49-81): a
# `functions` string with doubled braces, abs() of a double, pow, M_PI
FUNCTIONS = """
    __device__ double E(double t)
    {{
        return -F * sin(omega * t) * pow(sin(omega * t / 16.), 2);
    }}
    """


def test_consts_are_emitted_like_the_reference():
    c = cexpr.cuda_consts(dict(X_gridDIM=512, dt=0.01, name="x", flag=True, K=lambda p: p))
    assert "const int X_gridDIM = 512;" in c
    assert "const double dt = 1.000000000000000e-02;" in c
    assert "const int flag = 1;" in c and "name" not in c and " K " not in c


def test_reference_style_expressions_compile():
    consts = cexpr.cuda_consts(dict(X_gridDIM=512, X_amplitude=150.0, dt=0.01, F=0.04, omega=0.05698, Ip=0.59))
    exprs = {
        "v": "-1. / sqrt(X * X + 1.37) + X * E(t)",
        "bx": "pow(abs(sin(0.5 * M_PI * (X + X_amplitude) / X_amplitude)"
              " * sin(0.5 * M_PI * (X_prime + X_amplitude) / X_amplitude)), dt * 0.05)",
        "rho0": "exp(-2.0 * (pow(X - 0.1, 2) + pow(X_prime - 0.1, 2)) + cuda_complex(0., 0.3 * (X - X_prime)))",
        "delta": "double(i == j)",
        "h": "K(P, t) + V(X, t)",
        "heaviside": "0.5 * (1 + int(signbit(X + Ip)))",
        "theta": "X_minus * X_plus + Theta * Lambda",
    }
    cexpr.check_source(cexpr.module_source(consts, FUNCTIONS, exprs, K="0.5 * P * P",
                                           V="-1. / sqrt(X * X + 1.37) + X * E(t)"))


def test_compile_errors_are_reported():
    with pytest.raises(FastWignerError, match="NVRTC"):
        cexpr.check_source(cexpr.module_source("", "", {"bad": "undefined_function(X)"}))
