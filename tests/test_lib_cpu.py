"""CPU-side checks of the C ABI: the library loads and exports every symbol
the public header declares (no compute calls: there is no GPU here)."""
import ctypes
import re
from pathlib import Path

import pytest

from fastwigner_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "fastwigner.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|long long|size_t|const char\*|void)\s+\*?(fw_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "fw_wigner_propagate" in syms and "fw_last_error" in syms


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.fail("libfastwigner.so is not built (run python -m fastwigner_b200.build)")
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert set(header_symbols()) <= set(_lib.exported_symbols())


def test_abi_version_and_error_path():
    lib = _lib.load()
    assert lib.fw_abi_version() == _lib.FW_ABI_VERSION
    out = _lib.c_vp()
    rc = lib.fw_wigner_plan_create(101, 128, 1, _lib.FW_F32, ctypes.byref(out))
    assert rc == 1  # FW_EINVAL (odd size, as the reference asserts), checked before any device work
    assert b"must be even" in lib.fw_last_error()
    rc = lib.fw_wigner_plan_create(128, 8192, 1, _lib.FW_F32, ctypes.byref(out))
    assert rc == 1  # beyond the largest transform length
    rc = lib.fw_rho_plan_create(100, 1, _lib.FW_F64, ctypes.byref(out))
    assert rc == 1  # density-matrix plans: powers of two only
    assert b"power of two" in lib.fw_last_error()
