"""The C-ABI library loads on a CPU-only host and exports every symbol that
include/gpufem.h declares; host-only entry points work without a GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gpufem.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from gpu_fem_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding prototypes every declared symbol
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_host_only_entry_points():
    from gpu_fem_b200 import _lib
    L = _lib.lib()
    assert L.gf_version().decode().startswith("gpufem-b200")
    assert L.gf_status_string(_lib.GF_ZERO_PIVOT).decode() == "zero pivot in ILU factorization"
    o = _lib.gf_solve_opts()
    L.gf_solve_opts_default(ctypes.byref(o))
    assert o.restart > 0 and o.rtol > 0


def test_invalid_arguments_rejected_without_device():
    from gpu_fem_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.gf_assembler_create(None, ctypes.byref(h)) == _lib.GF_INVALID_ARG
    assert L.gf_add_residual(None, None, 0, None) == _lib.GF_INVALID_ARG
    assert L.gf_gmres_solve(None, None, None, None, None, None, None, None) == _lib.GF_INVALID_ARG
