"""The C-ABI library loads without a GPU and exports every symbol that
include/curfp.h declares; enum values equal the reference's."""
import ctypes
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "curfp.h").read_text()
    return sorted(set(re.findall(r"curfpStatus_t\s+(curfp\w+)\s*\(", text)))


def test_header_enums():
    text = (ROOT / "include" / "curfp.h").read_text()
    for name, val in [("CURFP_STATUS_SUCCESS", 0), ("CURFP_STATUS_NOT_INITIALIZED", 1),
                      ("CURFP_STATUS_ALLOC_FAILED", 2), ("CURFP_STATUS_INVALID_VALUE", 3),
                      ("CURFP_STATUS_EXECUTION_FAILED", 4), ("CURFP_OP_N", 0),
                      ("CURFP_OP_T", 1), ("CURFP_FILL_MODE_LOWER", 0),
                      ("CURFP_FILL_MODE_UPPER", 1)]:
        assert re.search(rf"{name}\s*=\s*{val}\b", text), name


def test_library_exports_header():
    from curfp_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    syms = declared_symbols()
    assert "curfpSpftrf" in syms and len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    from curfp_b200 import _lib
    assert set(_lib.SIGNATURES) <= set(syms)


def test_header_compiles_as_c():
    src = '#include "curfp.h"\nint main(void){curfpHandle_t h=0;(void)h;return 0;}\n'
    r = subprocess.run(["gcc", "-x", "c", "-fsyntax-only", "-I", str(ROOT / "include"),
                        "-I", "/usr/local/cuda/include", "-"], input=src, text=True,
                       capture_output=True)
    assert r.returncode == 0, r.stderr


def test_python_api_surface():
    import curfp_b200 as c
    for name in ["ssfrk", "ssfrk_raw", "spftrf", "spftrf_raw", "spftrs", "spftrs_raw",
                 "spftri", "spftri_raw", "strttf", "strttf_raw", "stfttr", "stfttr_raw",
                 "ssfr2k", "ssfr2k_raw", "rfp_diag_indices", "add_to_diagonal",
                 "Handle", "set_stream"]:
        assert callable(getattr(c, name)), name
    assert (c.OP_N, c.OP_T, c.FILL_LOWER, c.FILL_UPPER) == (0, 1, 0, 1)


def test_torch_extension_registers_ops():
    """The torch extension (curfp_b200/csrc_torch/torch_ops.cpp) loads on a
    machine without a GPU and registers every operator the autograd layer
    calls."""
    import torch

    from curfp_b200._torch_ops import ops
    o = ops()
    for name in ("ssfrk", "add_to_diagonal", "spftrf", "spftrs", "spftrs_refine",
                 "ssfrk_backward", "spftrf_backward", "spftrs_backward", "gpnll_backward"):
        assert hasattr(o, name), name
        assert "curfp_b200::" + name in str(getattr(o, name).default._schema)
