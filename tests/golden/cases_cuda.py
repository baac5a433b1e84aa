"""Cases of the reference's CUDA-class fixtures (tests/golden/gen_golden_cuda.py).

Every case is a set of constructor keywords with C-string Hamiltonians, as
the reference's CUDA classes take them (the drop-in classes take the same
strings), an initial state given as a C string (or the class's own delta /
W = const start for the Bloch runs), and what to run.  Grids are small so the
reference kernels, compiled for the host, run in seconds.
"""

_DW = dict(K="0.5 * P * P", V="0.05 * X * X * X * X - X * X", diff_K="P", diff_V="0.2 * X * X * X - 2.0 * X")
_FIELD_FN = "__device__ double E(double t){ return -F * sin(omega * t) * pow(sin(omega * t / 16.), 2); }"

CUDA_CASES = {
    # von Neumann, double well, Ehrenfest lists + Wigner time (Ip), 25 steps
    "rho_vn_dw_128": dict(
        cls="RhoVNeumannCUDA1D",
        kw=dict(t=0.0, dt=0.005, X_gridDIM=128, X_amplitude=10.0, Ip=0.4, **_DW),
        init="exp(-1.5 * (pow(X - 0.7, 2) + pow(X_prime - 0.7, 2)) + cuda_complex(0., -0.3 * (X - X_prime)))",
        steps=25, wigner_time=True),
    # von Neumann, time-dependent length-gauge field from a `functions` string,
    # both absorbing boundaries, C-string complex initial state
    "rho_vn_field_abs_128": dict(
        cls="RhoVNeumannCUDA1D",
        kw=dict(t=5.0, dt=0.02, X_gridDIM=128, X_amplitude=10.0, F=0.2, omega=0.3, Ip=0.5, functions=_FIELD_FN,
                K="0.5 * P * P", V="-1. / sqrt(X * X + 1.37) + X * E(t)", diff_K="P",
                diff_V="X / pow(X * X + 1.37, 1.5) + E(t)",
                abs_boundary_x="pow(abs(sin(0.5 * M_PI * (X + X_amplitude) / X_amplitude)"
                               " * sin(0.5 * M_PI * (X_prime + X_amplitude) / X_amplitude)), dt * 0.05)",
                abs_boundary_p="exp(-1e-3 * dt * (P * P + P_prime * P_prime))"),
        init="exp(-2.0 * (pow(X - 0.5, 2) + pow(X_prime - 0.5, 2)) + cuda_complex(0., 0.4 * (X - X_prime)))",
        steps=15, wigner_time=True),
    # Bloch rho: Gibbs state of the double well from the delta start (K_min = 0 as in the reference)
    "rho_bloch_gibbs_dw_128": dict(
        cls="RhoBlochCUDA1D",
        kw=dict(t=0.0, X_gridDIM=128, X_amplitude=8.0, dbeta=0.01, K="0.5 * P * P",
                V="0.05 * X * X * X * X - X * X"),
        gibbs=dict(kT=0.5, dbeta=0.01)),
    # Bloch rho: ground state with roll-back and dbeta halving (harmonic)
    "rho_bloch_ground_harmonic_128": dict(
        cls="RhoBlochCUDA1D",
        kw=dict(t=0.0, X_gridDIM=128, X_amplitude=8.0, dbeta=0.05, K="0.5 * P * P", V="0.5 * X * X"),
        ground=dict(dbeta=0.1, abs_tol_purity=1e-9)),
    # Moyal, CUDA convention: field, all three absorbing boundaries, C-string init
    "wigner_cuda_field_abs_256x128": dict(
        cls="WignerMoyalCUDA1D",
        kw=dict(t=3.0, dt=0.02, X_gridDIM=256, X_amplitude=12.0, P_gridDIM=128, P_amplitude=6.0, F=0.3, omega=0.7,
                functions=_FIELD_FN, K="0.5 * P * P", V="-1. / sqrt(X * X + 1.37) + X * E(t)", diff_K="P",
                diff_V="X / pow(X * X + 1.37, 1.5) + E(t)",
                abs_boundary_x_theta="exp(-1e-4 * Theta * Theta)",
                abs_boundary_lambda_p="exp(-1e-4 * Lambda * Lambda)",
                abs_boundary_x_p="pow(abs(sin(0.5 * M_PI * (X + X_amplitude) / X_amplitude)), dt * 0.5)"),
        init="exp(-(X - 1.0) * (X - 1.0) - 2.0 * P * P)",
        steps=15),
    # Bloch W (CUDA class): Gibbs state of the double well
    "wigner_bloch_cuda_dw_128": dict(
        cls="WignerBlochCUDA1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0, t_initial=0.0,
                K="0.5 * P * P", V="0.05 * X * X * X * X - X * X"),
        gibbs=dict(kT=0.5, dbeta=0.01)),
    # Bloch W (CUDA class): ground state with roll-back and dbeta halving (harmonic;
    # the double well's near-degenerate lowest pair converges far too slowly)
    "wigner_bloch_cuda_ground_harmonic_128": dict(
        cls="WignerBlochCUDA1D",
        kw=dict(t=0.0, dt=0.01, X_gridDIM=128, X_amplitude=8.0, P_gridDIM=128, P_amplitude=7.0, t_initial=0.0,
                K="0.5 * P * P", V="0.5 * X * X"),
        ground=dict(dbeta=0.05, abs_tol_purity=1e-9)),
}
