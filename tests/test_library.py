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


def _desc(conn, xpts, bcs, data, nn=None):
    from gpu_fem_b200 import _lib
    d = _lib.gf_mesh_desc()
    d.num_nodes = nn if nn is not None else len(xpts) // 3
    d.num_elements = len(conn) // 4
    d.conn = conn.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    d.xpts = xpts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.bcs = bcs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if len(bcs) else None
    d.num_bcs = len(bcs)
    d.data = ctypes.cast(data, ctypes.POINTER(_lib.gf_shell_data))
    d.ordering = _lib.GF_ORDER_NATURAL
    return d


def test_malformed_meshes_rejected_before_any_device_work():
    """Empty, ragged and out-of-range inputs are refused with GF_INVALID_ARG
    (validated on the host, before a device is looked up): no elements, a
    node index past the node count, a repeated node in an element, a
    negative node, and a constrained DOF past 6 x nodes."""
    import numpy as np
    from gpu_fem_b200 import _lib
    L = _lib.lib()
    xpts = np.zeros(12)
    data = (_lib.gf_shell_data * 1)()
    h = ctypes.c_void_p()
    ok_conn = np.array([0, 1, 2, 3], np.int32)
    none = np.zeros(0, np.int32)
    cases = {
        "no elements": _desc(np.zeros(0, np.int32), xpts, none, data),
        "node past the count": _desc(np.array([0, 1, 2, 4], np.int32), xpts, none, data),
        "repeated node": _desc(np.array([0, 1, 1, 3], np.int32), xpts, none, data),
        "negative node": _desc(np.array([0, -1, 2, 3], np.int32), xpts, none, data),
        "BC past 6 x nodes": _desc(ok_conn, xpts, np.array([24], np.int32), data),
        "no nodes": _desc(ok_conn, xpts, none, data, nn=0),
    }
    for name, d in cases.items():
        assert L.gf_assembler_create(ctypes.byref(d), ctypes.byref(h)) == _lib.GF_INVALID_ARG, name


def test_bdf_reader_errors_without_device(tmp_path):
    """BDF input errors are host-side status codes with a text: a missing
    file, an element on a missing GRID, an SPC on a missing GRID."""
    from gpu_fem_b200 import _lib
    L = _lib.lib()
    m = ctypes.POINTER(_lib.gf_bdf_mesh)()
    assert L.gf_bdf_read(str(tmp_path / "absent.bdf").encode(), ctypes.byref(m)) == _lib.GF_INVALID_ARG
    assert b"cannot open" in L.gf_last_error()
    p = tmp_path / "bad.bdf"
    p.write_text("BEGIN BULK\nGRID,1,0,0.,0.,0.\nGRID,2,0,1.,0.,0.\nGRID,3,0,1.,1.,0.\n"
                 "CQUAD4,1,1,1,2,3,9\nENDDATA\n")
    assert L.gf_bdf_read(str(p).encode(), ctypes.byref(m)) == _lib.GF_INVALID_ARG
    assert b"missing GRID" in L.gf_last_error()
    p.write_text("BEGIN BULK\nGRID,1,0,0.,0.,0.\nSPC,1,7,123\nENDDATA\n")
    assert L.gf_bdf_read(str(p).encode(), ctypes.byref(m)) == _lib.GF_INVALID_ARG
    assert b"SPC on missing GRID" in L.gf_last_error()
