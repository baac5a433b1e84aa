"""ctypes binding of libfastwigner.so (the C ABI declared in include/fastwigner.h).

The library is built in-tree (``python -m fastwigner_b200.build``).  There is
no CPU fallback: if the library or a CUDA device is missing, every entry
point raises ``FastWignerError``.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().with_name("libfastwigner.so")

FW_F32, FW_F64 = 0, 1
FW_STEP_FUSED, FW_STEP_SPLIT = 0, 1
FW_ABI_VERSION = 1


class FastWignerError(RuntimeError):
    """A libfastwigner call failed (the message comes from fw_last_error)."""


c_vp = ctypes.c_void_p
c_ll = ctypes.c_longlong
c_int = ctypes.c_int
c_dbl = ctypes.c_double


class WignerDesc(ctypes.Structure):
    """Mirror of ``fw_wigner_desc`` (include/fastwigner.h)."""

    _fields_ = [
        ("W", c_vp), ("w_bstride", c_ll), ("step_kind", c_int),
        ("tabV", c_vp), ("tabV_step", c_ll), ("tabK", c_vp), ("tabK_step", c_ll),
        ("tab_bstride", c_ll), ("tab_real", c_int),
        ("gV", c_vp), ("gV_step", c_ll), ("gK", c_vp), ("gK_step", c_ll),
        ("bxp", c_vp), ("bxp_bstride", c_ll),
        ("s0", c_vp), ("s0_bstride", c_ll), ("blend_c", c_dbl),
        ("Mx", c_int), ("Mp", c_int),
        ("wx", c_vp), ("wx_step", c_ll), ("wx_bstride", c_ll),
        ("wp", c_vp), ("wp_step", c_ll), ("wp_bstride", c_ll),
        ("obs_out", c_vp), ("dxdp", c_dbl), ("in_scale", c_dbl),
    ]


class RhoFactor(ctypes.Structure):
    """Mirror of ``fw_rho_factor``."""

    _fields_ = [("on", c_int), ("s_re", c_dbl), ("s_im", c_dbl), ("u", c_vp), ("w", c_vp), ("tab", c_vp),
                ("tab_bstride", c_ll), ("shear_c", c_dbl), ("shear_a", c_int), ("shear_b", c_int),
                ("shear_dx", c_dbl), ("shear_dp", c_dbl), ("sign", c_int)]


class RhoDesc(ctypes.Structure):
    """Mirror of ``fw_rho_desc``."""

    _fields_ = [("R", c_vp), ("r_bstride", c_ll), ("uV", c_vp), ("wV", c_vp), ("V_step", c_ll),
                ("uK", c_vp), ("wK", c_vp), ("K_step", c_ll), ("bx", c_vp), ("bp", c_vp), ("b_bstride", c_ll),
                ("Mx", c_int), ("Mp", c_int), ("wx", c_vp), ("wx_step", c_ll), ("gp", c_vp), ("gp_step", c_ll),
                ("obs_out", c_vp), ("dX", c_dbl)]


# (name, restype, argtypes) of every exported entry point
_SIGNATURES = [
    ("fw_abi_version", c_int, []),
    ("fw_last_error", ctypes.c_char_p, []),
    ("fw_wigner_plan_create", c_int, [c_int, c_int, c_int, c_int, ctypes.POINTER(c_vp)]),
    ("fw_wigner_plan_destroy", c_int, [c_vp]),
    ("fw_wigner_num_obs", c_int, [c_int, c_int]),
    ("fw_wigner_plan_status", c_int, [c_vp, ctypes.POINTER(c_int), c_int]),
    ("fw_wigner_propagate", c_int, [c_vp, ctypes.POINTER(WignerDesc), c_int, c_vp]),
    ("fw_wigner_weighted_sum", c_int, [c_vp, c_vp, c_ll, c_vp, c_vp, c_vp]),
    ("fw_wigner_propagate_timed", c_int, [c_vp, ctypes.POINTER(WignerDesc), c_int, c_vp,
                                          ctypes.POINTER(ctypes.c_float), ctypes.POINTER(c_int), c_int]),
    ("fw_launch_count", c_ll, []),
    ("fw_wigner_propagate_noalloc", c_int, [c_int, c_int, c_int, c_int, ctypes.POINTER(WignerDesc), c_int, c_vp]),
    ("fw_noalloc_scratch_bytes", ctypes.c_size_t, []),
    ("fw_noalloc_scratch_needed", ctypes.c_size_t, [c_int, c_int, c_int, c_int, ctypes.POINTER(WignerDesc)]),
    ("fw_rho_plan_create", c_int, [c_int, c_int, c_int, ctypes.POINTER(c_vp)]),
    ("fw_rho_plan_destroy", c_int, [c_vp]),
    ("fw_rho_num_parts", c_int, [c_vp]),
    ("fw_rho_pass", c_int, [c_vp, c_vp, c_ll, c_int, ctypes.POINTER(RhoFactor), c_int, ctypes.POINTER(RhoFactor),
                            ctypes.POINTER(RhoFactor), c_int, ctypes.POINTER(RhoFactor), c_vp, c_vp, c_vp]),
    ("fw_rho_propagate", c_int, [c_vp, ctypes.POINTER(RhoDesc), c_int, c_vp]),
    ("fw_batch_create", c_int, [c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_int, ctypes.POINTER(c_vp)]),
    ("fw_batch_destroy", c_int, [c_vp]),
    ("fw_batch_num_variants", c_int, []),
    ("fw_batch_set_variant", c_int, [c_vp, c_int]),
    ("fw_batch_set_instance", c_int, [c_vp, c_int, c_vp, c_vp, c_vp, c_dbl]),
    ("fw_batch_propagate", c_int, [c_vp, c_int, c_vp, c_int, c_vp]),
    ("fw_batch_status", c_int, [c_vp, ctypes.POINTER(c_int)]),
    ("fw_batch_set_status", c_int, [c_vp, c_int]),
    ("fw_batch_set_spin_limit", c_int, [c_vp, c_ll]),
    ("fw_fno_sgemm", c_int, [c_int, c_int, c_int, c_int, c_int, ctypes.c_float, c_vp, c_ll, c_ll, c_vp, c_ll, c_ll,
                              ctypes.c_float, c_vp, c_ll, c_ll, c_int, c_vp]),
    ("fw_fno_sgemm_ex", c_int, [c_int, c_int, c_int, c_int, c_int, ctypes.c_float, c_vp, c_ll, c_ll, c_vp, c_ll, c_ll,
                                ctypes.c_float, c_vp, c_ll, c_ll, c_int, c_vp, c_vp, c_vp, c_int, c_vp, c_vp]),
    ("fw_fno_wgrad_work", c_int, [c_int, c_int, c_ll, c_int, ctypes.POINTER(c_ll)]),
    ("fw_fno_wgrad", c_int, [c_int, c_int, c_ll, c_vp, c_ll, c_vp, c_ll, c_int, c_vp, c_ll, c_vp, c_int, c_vp]),
    ("fw_fno_project", c_int, [c_int, c_int, c_ll, c_vp, c_ll, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_ll, c_vp]),
    ("fw_fno_status", c_int, [ctypes.POINTER(c_int), c_int]),
    ("fw_fno_mix", c_int, [c_int, c_int, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    ("fw_fno_bias_act", c_int, [c_ll, c_int, c_ll, c_vp, c_vp, c_vp, c_vp, c_int, c_vp]),
    ("fw_fno_act_bwd", c_int, [c_ll, c_vp, c_vp, c_vp, c_int, c_vp]),
    ("fw_fno_channel_sum", c_int, [c_int, c_int, c_ll, c_vp, c_vp, c_int, c_vp]),
    ("fw_fno_rel_l2", c_int, [c_int, c_ll, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fw_fno_adam", c_int, [c_ll, c_vp, c_vp, c_vp, c_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                            ctypes.c_float, c_int, ctypes.c_float, c_vp]),
    ("fw_fno_features", c_int, [c_int, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fw_expr_create", c_int, [ctypes.c_char_p, ctypes.POINTER(c_vp)]),
    ("fw_expr_destroy", c_int, [c_vp]),
    ("fw_expr_check", c_int, [ctypes.c_char_p, ctypes.c_char_p, c_int]),
    ("fw_expr_eval", c_int, [c_vp, ctypes.c_char_p, c_vp, c_ll, c_vp, c_vp, c_vp]),
]

_lib = None


def load() -> ctypes.CDLL:
    """Load libfastwigner.so (once) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FastWignerError(
            f"{LIB_PATH.name} is not built; run `python -m fastwigner_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, res, args in _SIGNATURES:
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if lib.fw_abi_version() != FW_ABI_VERSION:
        raise FastWignerError("libfastwigner ABI version mismatch; rebuild the library")
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = load().fw_last_error().decode(errors="replace")
        raise FastWignerError(f"{what}: {msg}" if what else msg)


def exported_symbols() -> list[str]:
    return [name for name, _, _ in _SIGNATURES]
