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


def test_params_struct_layout_matches_header(tmp_path):
    """The ctypes mirror of ckks_params has the C struct's size and field
    offsets (a C program built against include/ckks_b200.h prints them)."""
    import ctypes
    import shutil
    import subprocess
    from pathlib import Path
    from ckks_b200._lib import CkksParamsC
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = Path(__file__).resolve().parents[1] / "include"
    fields = [f for f, _ in CkksParamsC._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ckks_b200.h"\nint main(void) {\n'
                   '  printf("%zu", sizeof(ckks_params));\n'
                   + "".join(f'  printf(" %zu", offsetof(ckks_params, {f}));\n' for f in fields)
                   + '  printf("\\n");\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(inc), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == [ctypes.sizeof(CkksParamsC)] + [getattr(CkksParamsC, f).offset for f in fields]
