"""ctypes binding of libgpufem.so (the C ABI declared in include/gpufem.h).

The library is built in-tree (gpu_fem_b200/libgpufem.so). There is no CPU
fallback: if the shared library is missing, importing the bound functions
raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpufem.so")

GF_OK, GF_INVALID_ARG, GF_OOM, GF_ZERO_PIVOT, GF_NOT_CONVERGED, GF_NAN, GF_TIMEOUT, \
    GF_CUDA_ERROR, GF_NO_DEVICE, GF_OVER_BUDGET = range(10)
GF_ORDER_NATURAL, GF_ORDER_RCM, GF_ORDER_QORDER = 0, 1, 2
GF_ASSEMBLE_OVERWRITE, GF_ASSEMBLE_ADD, GF_ASSEMBLE_FUSE_BCS, GF_ASSEMBLE_ATOMIC = 0, 1, 2, 4
GF_PREC_FP64, GF_PREC_FP32 = 0, 1
GF_SWEEP_AUTO, GF_SWEEP_DATAFLOW, GF_SWEEP_LEVEL = 0, 1, 2
GF_FILL_FULL = 0x7FFFFFFF


class GpuFemError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = lib().gf_status_string(status).decode()
        last = lib().gf_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}){' — ' + last if last else ''}")


class gf_shell_data(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("thick", C.c_double),
                ("tOffset", C.c_double), ("refAxis", C.c_double * 3),
                ("has_ref_axis", C.c_int32), ("pad", C.c_int32)]


class gf_mesh_desc(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_elements", C.c_int32),
                ("conn", C.POINTER(C.c_int32)), ("xpts", C.POINTER(C.c_double)),
                ("bcs", C.POINTER(C.c_int32)), ("num_bcs", C.c_int32),
                ("data", C.POINTER(gf_shell_data)), ("ordering", C.c_int32),
                ("rcm_root", C.c_int32), ("qorder_p", C.c_double), ("qorder_seed", C.c_uint64)]


class gf_solve_opts(C.Structure):
    _fields_ = [("restart", C.c_int32), ("max_iters", C.c_int32), ("rtol", C.c_double),
                ("side", C.c_int32), ("mixed", C.c_int32), ("inner_rtol", C.c_double),
                ("max_refine", C.c_int32), ("check_every", C.c_int32)]


class gf_solve_stats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("restarts", C.c_int32),
                ("refinements", C.c_int32), ("status", C.c_int32),
                ("rel_residual", C.c_double), ("time_ms", C.c_double)]


class gf_bdf_mesh(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_elements", C.c_int32), ("num_bcs", C.c_int32),
                ("conn", C.POINTER(C.c_int32)), ("xpts", C.POINTER(C.c_double)),
                ("bcs", C.POINTER(C.c_int32)), ("component", C.POINTER(C.c_int32)),
                ("impl", C.c_void_p)]


_P = C.c_void_p
_I = C.c_int32
_D = C.c_double
_PI = C.POINTER(C.c_int32)
_PU = C.POINTER(C.c_uint32)
_PD = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol include/gpufem.h declares
SIGNATURES = {
    "gf_status_string": (C.c_char_p, [_I]),
    "gf_version": (C.c_char_p, []),
    "gf_last_error": (C.c_char_p, []),
    "gf_launch_count": (C.c_longlong, []),
    "gf_assembler_create": (_I, [C.POINTER(gf_mesh_desc), C.POINTER(_P)]),
    "gf_assembler_destroy": (_I, [_P]),
    "gf_order_nodes": (_I, [C.POINTER(gf_mesh_desc), _PI]),
    "gf_assembler_num_nodes": (_I, [_P]),
    "gf_assembler_num_elements": (_I, [_P]),
    "gf_assembler_num_vars": (_I, [_P]),
    "gf_assembler_nnzb": (_I, [_P]),
    "gf_assembler_get_pattern": (_I, [_P, _PI, _PI, _PI, _PI]),
    "gf_assembler_get_schedule": (_I, [_P, _PI, _PI, _PI, _PU, _PI, _PI]),
    "gf_set_variables": (_I, [_P, _P, _P]),
    "gf_assembler_set_thickness": (_I, [_P, _P, _P]),
    "gf_add_residual": (_I, [_P, _P, _I, _P]),
    "gf_add_jacobian": (_I, [_P, _P, _P, _I, _P]),
    "gf_add_jacobian_thick": (_I, [_P, _P, _P, _P, _I, _P]),
    "gf_add_energy": (_I, [_P, _PD, _P]),
    "gf_apply_bcs_vec": (_I, [_P, _P, _P]),
    "gf_apply_bcs_mat": (_I, [_P, _P, _P]),
    "gf_bsr_create": (_I, [_P, C.POINTER(_P)]),
    "gf_bsr_destroy": (_I, [_P]),
    "gf_bsr_values": (_P, [_P]),
    "gf_bsr_zero": (_I, [_P, _P]),
    "gf_bsr_spmv": (_I, [_P, _D, _P, _D, _P, _P]),
    "gf_permute_vec": (_I, [_P, _P, _P, _I, _P]),
    "gf_precond_create": (_I, [_P, _I, _I, C.POINTER(_P)]),
    "gf_precond_create_ex": (_I, [_P, _I, _I, _I, C.POINTER(_P)]),
    "gf_precond_sweeps": (_I, [_P, _PI, _PI, _PI, _PI]),
    "gf_precond_destroy": (_I, [_P]),
    "gf_precond_factor": (_I, [_P, _P, _P]),
    "gf_precond_apply": (_I, [_P, _P, _P, _P]),
    "gf_precond_apply_noalloc": (_I, [_P, _P, _P, _P]),
    "gf_timing_enable": (_I, [C.c_int32]),
    "gf_timing_read": (_I, [C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                            C.POINTER(C.c_double)]),
    "gf_precond_info": (_I, [_P, _PI, _PI, _PI]),
    "gf_precond_status": (_I, [_P, _P]),
    "gf_precond_layout": (_I, [_P, _PI, _PI, _PI, _PI, _PI]),
    "gf_batch_set_scatter": (_I, [_P, C.c_int32]),
    "gf_assembler_setup_info": (_I, [_P, _PI, _PI]),
    "gf_precond_setup_info": (_I, [_P, _PI, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "gf_test_set_waits": (_I, [C.c_ulonglong, _I]),
    "gf_precond_get": (_I, [_P, _PI, _PI, _PD]),
    "gf_solve_opts_default": (None, [C.POINTER(gf_solve_opts)]),
    "gf_gmres_solve": (_I, [_P, _P, _P, _P, _P, C.POINTER(gf_solve_opts),
                            C.POINTER(gf_solve_stats), _P]),
    "gf_direct_solve": (_I, [_P, _P, _P, _P, C.POINTER(gf_solve_stats), _P]),
    "gf_bdf_read": (_I, [C.c_char_p, C.POINTER(C.POINTER(gf_bdf_mesh))]),
    "gf_bdf_free": (_I, [C.POINTER(gf_bdf_mesh)]),
    "gf_batch_create": (_I, [_I, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "gf_batch_destroy": (_I, [_P]),
    "gf_batch_assemble": (_I, [_P, _P]),
    "gf_batch_assemble_ex": (_I, [_P, C.POINTER(_P), _P]),
    "gf_batch_factor": (_I, [_P, _P]),
    "gf_batch_solve": (_I, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(gf_solve_opts),
                            C.POINTER(gf_solve_stats), _P]),
}

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgpufem.so not built at {LIB_PATH}; run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(status, where=""):
    if status != GF_OK:
        raise GpuFemError(status, where)
    return status
