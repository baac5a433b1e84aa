"""Parity cases shared by the golden-fixture generator and the tests.

Each case is a dict of reference-class keyword arguments (Python callables,
as the reference's FFTW classes take them) plus a run recipe.  Sizes are
small enough for the FP64 oracle to finish in seconds.
"""
import numpy as np


def coherent(x0, p0, s=1.0):
    return lambda self, x, p: np.exp(-s * (x - x0) ** 2 - (p - p0) ** 2 / s) / np.pi + 0 * x * p


F_LASER, OMEGA_LASER = 0.04, 0.05698


def vector_potential(t):
    """A(t) of strong_field_physics_fftw_1d.py:63."""
    return -F_LASER / OMEGA_LASER * np.sin(OMEGA_LASER * t) * np.sin(OMEGA_LASER * t / 16.0) ** 2


HARMONIC = dict(
    K=lambda _, p: 0.5 * p ** 2,
    V=lambda _, x: 0.5 * x ** 2,
    diff_K=lambda _, p: p,
    diff_V=lambda _, x: x,
)

DOUBLE_WELL = dict(
    K=lambda _, p: 0.5 * p ** 2,
    V=lambda _, x: 0.05 * x ** 4 - x ** 2,
    diff_K=lambda _, p: p,
    diff_V=lambda _, x: 0.2 * x ** 3 - 2.0 * x,
)

VELOCITY_GAUGE = dict(
    K=lambda _, p, t: 0.5 * (p + vector_potential(t)) ** 2,
    diff_K=lambda _, p, t: p + vector_potential(t),
    V=lambda _, x: -0.37 * (1 + np.cos(2 * np.pi * x / 8.0)),
    diff_V=lambda _, x: 0.37 * 2 * np.pi / 8.0 * np.sin(2 * np.pi * x / 8.0),
)

CASES = {
    # config-1 shape (harmonic, coherent state) on a 128^2 grid
    "moyal_harmonic_128": dict(
        cls="WignerMoyalFTTW1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0, **HARMONIC),
        init=coherent(1.0, 0.5), steps=20),
    # anharmonic double well, non-square grid, absorbing boundary (alpha)
    "moyal_dw_alpha_128x256": dict(
        cls="WignerMoyalFTTW1D",
        kw=dict(t=0.0, dt=0.005, X_gridDIM=256, X_amplitude=10.0, P_gridDIM=128, P_amplitude=10.0, alpha=0.5,
                **DOUBLE_WELL),
        init=coherent(-1.3, 0.4, 0.5), steps=30),
    # time-dependent kinetic energy (velocity gauge), Mathieu lattice
    "moyal_velocity_gauge_128x256": dict(
        cls="WignerMoyalFTTW1D",
        kw=dict(t=150.0, dt=0.05, X_gridDIM=256, X_amplitude=8.0, P_gridDIM=128, P_amplitude=10.0,
                **VELOCITY_GAUGE),
        init=coherent(0.0, 0.0, 1.0), steps=25),
    # FFTW Bloch Gibbs state (note: the reference's FFTW exponents give exp(-2H/kT))
    "bloch_fftw_harmonic_128": dict(
        cls="WignerBlochFFTW1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0, kT=0.5,
                dbeta=0.01, K=lambda _, p: 0.5 * p ** 2, V=lambda _, x: 0.5 * x ** 2)),
    # random-collision dephasing around a harmonic Moyal step
    "collision_harmonic_128": dict(
        cls="WignerRandomCollisionModelFFTW1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0, gamma=0.5, kT=0.5,
                **HARMONIC),
        init=coherent(1.5, -0.5), steps=20),
    # even sizes that are not powers of two (the reference only asserts evenness):
    # 96 = 4^2 2 3, 192 = 4^3 3, 100 = 4 5^2, 160 = 4^2 2 5, 98 = 2 7^2, 202 = 2 101
    "moyal_dw_96x192": dict(
        cls="WignerMoyalFTTW1D",
        kw=dict(t=0.0, dt=0.005, X_gridDIM=192, X_amplitude=10.0, P_gridDIM=96, P_amplitude=10.0, **DOUBLE_WELL),
        init=coherent(-1.3, 0.4, 0.5), steps=30),
    "moyal_harmonic_100": dict(
        cls="WignerMoyalFTTW1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=100, X_amplitude=8.0, P_gridDIM=100, P_amplitude=7.0, **HARMONIC),
        init=coherent(1.0, 0.5), steps=20),
    "moyal_dw_98x202": dict(
        cls="WignerMoyalFTTW1D",
        kw=dict(t=0.0, dt=0.005, X_gridDIM=202, X_amplitude=10.0, P_gridDIM=98, P_amplitude=10.0, alpha=0.5,
                **DOUBLE_WELL),
        init=coherent(0.8, -0.3, 0.5), steps=15),
    "bloch_fftw_harmonic_160": dict(
        cls="WignerBlochFFTW1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=160, X_amplitude=8.0, P_gridDIM=160, P_amplitude=7.0, kT=0.5,
                dbeta=0.01, K=lambda _, p: 0.5 * p ** 2, V=lambda _, x: 0.5 * x ** 2)),
    "collision_harmonic_96": dict(
        cls="WignerRandomCollisionModelFFTW1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=96, X_amplitude=8.0, P_gridDIM=96, P_amplitude=7.0, gamma=0.5, kT=0.5,
                **HARMONIC),
        init=coherent(1.5, -0.5), steps=20),
}

# The configuration-1 workload at full size; only observables are stored.
CONFIG1 = dict(
    cls="WignerMoyalFTTW1D",
    kw=dict(t=0.0, dt=0.01, X_gridDIM=256, X_amplitude=8.0, P_gridDIM=256, P_amplitude=7.0, **HARMONIC),
    init=coherent(1.0, 0.5), steps=1000)
