"""The C-ABI library loads and exports every entry point the header declares
(no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ckks_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ckks_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_core_entries():
    syms = declared_symbols()
    for s in ("ckks_ctx_create", "ckks_ntt", "ckks_ct_mul_relin_rescale", "ckks_rescale_exact",
              "ckks_relin_single", "ckks_poly_mul"):
        assert s in syms


def test_library_exports_all_declared_symbols():
    from ckks_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.fail(f"{_lib.LIB_PATH} not built (run cipher-pu_b200/build.py)")
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_table_matches_header():
    from ckks_b200 import _lib
    assert set(_lib.SIGNATURES) == set(declared_symbols())


def test_error_channel_without_gpu():
    from ckks_b200 import _lib
    lib = _lib.load()
    assert lib.ckks_abi_version() >= 1
    # argument validation happens before any device work
    rc = lib.ckks_rescale_exact(None, None, -1, 5, 3, None)
    assert rc == 1
    assert b"n < 0" in lib.ckks_last_error()
