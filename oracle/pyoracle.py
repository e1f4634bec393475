"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() (as the checker) and
bench.py's CPU-baseline leg load this module. The product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class ShellData(C.Structure):
    """Mirrors ShellIsotropicData (include/shell/data.h:8-47)."""
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("thick", C.c_double),
                ("tOffset", C.c_double), ("refAxis", C.c_double * 3),
                ("has_ref_axis", C.c_int)]


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.orc_element_energy.restype = C.c_double
        _LIB.orc_assemble_energy.restype = C.c_double
    return _LIB


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def _pi(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def make_data(E, nu, thick, tOffset=0.0, ref_axis=None):
    d = ShellData()
    d.E, d.nu, d.thick, d.tOffset = E, nu, thick, tOffset
    if ref_axis is not None:
        for i in range(3):
            d.refAxis[i] = ref_axis[i]
        d.has_ref_axis = 1
    else:
        d.has_ref_axis = 0
    return d


def data_array(E, nu, thick):
    thick = np.asarray(thick, dtype=np.float64)
    arr = (ShellData * len(thick))()
    for i, t in enumerate(thick):
        arr[i].E, arr[i].nu, arr[i].thick, arr[i].tOffset = E, nu, float(t), 0.0
        arr[i].has_ref_axis = 0
    return arr


def element_residual(X, u, d):
    X = np.ascontiguousarray(X, np.float64).ravel()
    u = np.ascontiguousarray(u, np.float64).ravel()
    r = np.zeros(24)
    lib().orc_element_residual(_p(X), _p(u), C.byref(d), _p(r))
    return r


def element_jacobian(X, u, d):
    X = np.ascontiguousarray(X, np.float64).ravel()
    u = np.ascontiguousarray(u, np.float64).ravel()
    r = np.zeros(24)
    K = np.zeros(576)
    lib().orc_element_jacobian(_p(X), _p(u), C.byref(d), _p(r), _p(K))
    return r, K.reshape(24, 24)


def element_energy(X, u, d):
    X = np.ascontiguousarray(X, np.float64).ravel()
    u = np.ascontiguousarray(u, np.float64).ravel()
    return lib().orc_element_energy(_p(X), _p(u), C.byref(d))


def element_energy_cs(X, u_re, u_im, d):
    X = np.ascontiguousarray(X, np.float64).ravel()
    a = np.ascontiguousarray(u_re, np.float64).ravel()
    b = np.ascontiguousarray(u_im, np.float64).ravel()
    re, im = C.c_double(), C.c_double()
    lib().orc_element_energy_cs(_p(X), _p(a), _p(b), C.byref(d), C.byref(re), C.byref(im))
    return complex(re.value, im.value)


def element_residual_cs(X, u_re, u_im, d):
    X = np.ascontiguousarray(X, np.float64).ravel()
    a = np.ascontiguousarray(u_re, np.float64).ravel()
    b = np.ascontiguousarray(u_im, np.float64).ravel()
    rr, ri = np.zeros(24), np.zeros(24)
    lib().orc_element_residual_cs(_p(X), _p(a), _p(b), C.byref(d), _p(rr), _p(ri))
    return rr + 1j * ri


def bsr_pattern(conn, nnodes):
    conn = np.ascontiguousarray(conn, np.int32)
    ne = conn.shape[0]
    rowp = np.zeros(nnodes + 1, np.int32)
    nnz = lib().orc_bsr_pattern(ne, nnodes, _pi(conn), _pi(rowp), None)
    cols = np.zeros(nnz, np.int32)
    lib().orc_bsr_pattern(ne, nnodes, _pi(conn), _pi(rowp), _pi(cols))
    return rowp, cols


def rcm(rowp, cols, root=0, iters=1):
    n = len(rowp) - 1
    out = np.zeros(n, np.int32)
    lib().orc_rcm(n, _pi(rowp), _pi(cols), root, iters, _pi(out))
    return out


def qorder(rowp, cols, rcm_perm, pfac=1.0, seed=0):
    """Deterministic q-ordering on top of an RCM order (perm[old] = new)."""
    n = len(rowp) - 1
    out = np.zeros(n, np.int32)
    rcm_perm = np.ascontiguousarray(rcm_perm, np.int32)
    lib().orc_qorder(n, _pi(rowp), _pi(cols), _pi(rcm_perm), C.c_double(pfac),
                     C.c_ulonglong(seed), _pi(out))
    return out


def permute_pattern(rowp, cols, perm):
    n = len(rowp) - 1
    r2 = np.zeros(n + 1, np.int32)
    c2 = np.zeros(len(cols), np.int32)
    perm = np.ascontiguousarray(perm, np.int32)
    lib().orc_permute_pattern(n, _pi(rowp), _pi(cols), _pi(perm), _pi(r2), _pi(c2))
    return r2, c2


def elem_ind_map(conn, rowp, cols, perm):
    conn = np.ascontiguousarray(conn, np.int32)
    perm = np.ascontiguousarray(perm, np.int32)
    m = np.zeros(16 * conn.shape[0], np.int32)
    lib().orc_elem_ind_map(conn.shape[0], _pi(conn), _pi(rowp), _pi(cols), _pi(perm), _pi(m))
    return m


def assemble_jacobian(mesh, vars_=None, perm=None, nthreads=1):
    nn = mesh.num_nodes
    perm = np.arange(nn, dtype=np.int32) if perm is None else np.ascontiguousarray(perm, np.int32)
    rowp0, cols0 = bsr_pattern(mesh.conn, nn)
    rowp, cols = permute_pattern(rowp0, cols0, perm)
    emap = elem_ind_map(mesh.conn, rowp, cols, perm)
    vals = np.zeros(36 * len(cols))
    res = np.zeros(6 * nn)
    data = data_array(mesh.E, mesh.nu, mesh.thick)
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    xpts = np.ascontiguousarray(mesh.xpts, np.float64)
    v = None if vars_ is None else np.ascontiguousarray(vars_, np.float64)
    lib().orc_assemble_jacobian(conn.shape[0], _pi(conn), _p(xpts),
                                None if v is None else _p(v), data, _pi(emap), _p(vals),
                                _p(res), nthreads)
    return rowp, cols, vals, res, perm


def assemble_residual(mesh, vars_):
    res = np.zeros(6 * mesh.num_nodes)
    data = data_array(mesh.E, mesh.nu, mesh.thick)
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    xpts = np.ascontiguousarray(mesh.xpts, np.float64)
    v = np.ascontiguousarray(vars_, np.float64)
    lib().orc_assemble_residual(conn.shape[0], _pi(conn), _p(xpts), _p(v), data, _p(res))
    return res


def apply_bcs_mat(rowp, cols, vals, perm, bcs, fast=False):
    n = len(rowp) - 1
    bcs = np.ascontiguousarray(bcs, np.int32)
    perm = np.ascontiguousarray(perm, np.int32)
    f = lib().orc_apply_bcs_mat_fast if fast else lib().orc_apply_bcs_mat
    f(n, _pi(rowp), _pi(cols), _pi(perm), len(bcs), _pi(bcs), _p(vals))


def full_fill_count(rowp, cols):
    return lib().orc_full_fill_count(len(rowp) - 1, _pi(rowp), _pi(cols))


def ilu0(rowp, cols, vals):
    LU = vals.copy()
    st = lib().orc_ilu0_factor(len(rowp) - 1, _pi(rowp), _pi(cols), _p(LU))
    return st, LU


def ilu0_apply(rowp, cols, LU, r):
    z = np.zeros_like(r)
    lib().orc_ilu0_apply(len(rowp) - 1, _pi(rowp), _pi(cols), _p(LU), _p(r), _p(z))
    return z


def spmv(rowp, cols, vals, x):
    y = np.zeros_like(x)
    lib().orc_spmv(len(rowp) - 1, _pi(rowp), _pi(cols), _p(vals), _p(x), _p(y))
    return y


def levels(rowp, cols, lower=True):
    n = len(rowp) - 1
    lv = np.zeros(n, np.int32)
    nl = lib().orc_levels(n, _pi(rowp), _pi(cols), 1 if lower else 0, _pi(lv))
    return nl, lv


def invert_diag(rowp, cols, LU):
    """Factor values with each diagonal block U_ii replaced by U_ii^-1."""
    out = np.array(LU, np.float64).reshape(-1, 6, 6)
    n = len(rowp) - 1
    rows = np.repeat(np.arange(n), np.diff(rowp))
    d = np.nonzero(cols == rows)[0]
    out[d] = np.linalg.inv(out[d])
    return out.ravel()


def gmres(rowp, cols, A, LU, b, m=50, rtol=1e-10, maxit=20000, side=0, x0=None, prowp=None,
          pcols=None, nthreads=1):
    """Restarted GMRES(m) on A (rowp, cols) with the block ILU factor LU (as
    returned by ilu0: U_ii on the diagonal) on its pattern (prowp, pcols;
    A's pattern when omitted)."""
    prowp = rowp if prowp is None else prowp
    pcols = cols if pcols is None else pcols
    LUd = invert_diag(prowp, pcols, LU)
    b = np.ascontiguousarray(b, np.float64)
    A = np.ascontiguousarray(A, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    it, rel = C.c_int(), C.c_double()
    st = lib().orc_gmres_k(len(rowp) - 1, _pi(rowp), _pi(cols), _p(A), _pi(prowp), _pi(pcols),
                           _p(LUd), _p(b), _p(x), m, C.c_double(rtol), maxit, side, nthreads,
                           C.byref(it), C.byref(rel))
    return st, x, it.value, rel.value


def solve_problem(mesh, perm, fill, restart=200, rtol=1e-8, maxit=20000, nthreads=1):
    """One compiled CPU solve of a shell mesh (pattern, assembly + BCs, ILU(fill),
    right-preconditioned GMRES). Returns (status, x natural order, iterations,
    relative residual, [setup, assembly, factor, gmres] seconds)."""
    conn = np.ascontiguousarray(mesh.conn, np.int32)
    xpts = np.ascontiguousarray(mesh.xpts, np.float64)
    bcs = np.ascontiguousarray(mesh.bcs, np.int32)
    loads = np.ascontiguousarray(mesh.loads, np.float64)
    perm = np.ascontiguousarray(perm, np.int32)
    data = data_array(mesh.E, mesh.nu, mesh.thick)
    x = np.zeros(6 * mesh.num_nodes)
    t = np.zeros(4)
    it, rel = C.c_int(), C.c_double()
    st = lib().orc_solve_problem(conn.shape[0], mesh.num_nodes, _pi(conn), _p(xpts), data,
                                 len(bcs), _pi(bcs), _p(loads), _pi(perm), fill, restart,
                                 C.c_double(rtol), maxit, nthreads, _p(x), C.byref(it),
                                 C.byref(rel), _p(t))
    return st, x, it.value, rel.value, t


def dense_solve(A, b):
    A = np.ascontiguousarray(A, np.float64).copy()
    x = np.ascontiguousarray(b, np.float64).copy()
    st = lib().orc_dense_solve(len(x), _p(A), _p(x))
    if st:
        raise RuntimeError(f"dense solve failed at pivot {st}")
    return x


def bsr_to_dense(rowp, cols, vals):
    n = len(rowp) - 1
    A = np.zeros((6 * n, 6 * n))
    V = vals.reshape(-1, 6, 6)
    for i in range(n):
        for jp in range(rowp[i], rowp[i + 1]):
            j = cols[jp]
            A[6 * i:6 * i + 6, 6 * j:6 * j + 6] = V[jp]
    return A


def iluk_pattern(rowp, cols, lev):
    n = len(rowp) - 1
    r2 = np.zeros(n + 1, np.int32)
    nnz = lib().orc_iluk_pattern(n, _pi(rowp), _pi(cols), lev, _pi(r2), None)
    c2 = np.zeros(nnz, np.int32)
    lib().orc_iluk_pattern(n, _pi(rowp), _pi(cols), lev, _pi(r2), _pi(c2))
    return r2, c2


def scatter_to_pattern(rowp, cols, vals, rowp2, cols2):
    """Copy A's blocks into a superset pattern (copyValuesTo, bsr_mat.h:145-193)."""
    out = np.zeros(36 * len(cols2))
    vals = np.ascontiguousarray(vals, np.float64)
    st = lib().orc_scatter_to_pattern(len(rowp) - 1, _pi(rowp), _pi(cols), _p(vals), _pi(rowp2),
                                      _pi(cols2), _p(out))
    if st:
        raise ValueError(f"row {st - 1} of A has a block outside the target pattern")
    return out


def ilu_apply_dinv(rowp, cols, LU, r):
    """z = U^-1 L^-1 r for factors whose diagonal blocks hold U_ii^-1."""
    z = np.zeros_like(r)
    LU = np.ascontiguousarray(LU, np.float64)
    r = np.ascontiguousarray(r, np.float64)
    lib().orc_ilu_apply_dinv(len(rowp) - 1, _pi(rowp), _pi(cols), _p(LU), _p(r), _p(z))
    return z


def ilu_backward_error(rowp, cols, LU, A, dinv=True):
    """max |(L U - A)_ij| over the pattern and max |A| (sparse block products)."""
    out = np.zeros(2)
    LU = np.ascontiguousarray(LU, np.float64)
    A = np.ascontiguousarray(A, np.float64)
    lib().orc_ilu_backward_error(len(rowp) - 1, _pi(rowp), _pi(cols), _p(LU), _p(A),
                                 1 if dinv else 0, _p(out))
    return out[0], out[1]
