"""Python mirror of the reference's assembler-level API over the C ABI.

Class and method names follow smdogroup/gpu_fem: ElementAssembler
(include/assembler.h:14-322), BsrMat + createBsrMat
(include/linalg/bsr_mat.h:9-357), DeviceVec / HostVec (include/linalg/vec.h),
ILUk_Preconditioner (include/linalg/precond.h:5-55). Device memory is held in
torch CUDA tensors; all compute goes through libgpufem.so.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import _lib as L
from ._lib import check

__all__ = ["ElementAssembler", "BsrMat", "DeviceVec", "HostVec", "ILUk_Preconditioner",
           "createBsrMat", "SolveOptions", "gmres_solve"]


def _ptr(t: torch.Tensor) -> int:
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class HostVec:
    """Host vector (HostVec<T>, include/linalg/vec.h:297-371)."""

    def __init__(self, data):
        self.data = np.ascontiguousarray(data)

    def getSize(self):
        return self.data.size

    def createDeviceVec(self):
        return DeviceVec(torch.from_numpy(self.data.copy()).cuda())


class DeviceVec:
    """Device vector (DeviceVec<T>, include/linalg/vec.h:146-295)."""

    def __init__(self, t):
        if isinstance(t, int):
            t = torch.zeros(t, dtype=torch.float64, device="cuda")
        self.t = t

    def getPtr(self):
        return _ptr(self.t)

    def getSize(self):
        return self.t.numel()

    def zeroValues(self):
        self.t.zero_()

    def copyValuesTo(self, other):
        other.t.copy_(self.t)

    def createHostVec(self):
        return HostVec(self.t.cpu().numpy())


class ElementAssembler:
    """ElementAssembler<T, ShellElementGroup, DeviceVec, BsrMat>.

    Built from a gpu_fem_b200.mesh.ShellMesh (or explicit arrays)."""

    def __init__(self, conn, xpts, bcs, thick, E=70e9, nu=0.3, ordering="natural",
                 rcm_root=0, tOffset=0.0, ref_axis=None, qorder_p=1.0, qorder_seed=0):
        """ordering: "natural", "rcm" or "qorder" (deterministic q-ordering:
        the RCM order shuffled within windows of bandwidth / qorder_p
        positions, seeded with qorder_seed)."""
        conn = np.ascontiguousarray(conn, np.int32).reshape(-1, 4)
        xpts = np.ascontiguousarray(xpts, np.float64).reshape(-1, 3)
        bcs = np.ascontiguousarray(bcs, np.int32).ravel()
        thick = np.broadcast_to(np.asarray(thick, np.float64), (conn.shape[0],))
        data = (L.gf_shell_data * conn.shape[0])()
        E_arr = np.broadcast_to(np.asarray(E, np.float64), (conn.shape[0],))
        nu_arr = np.broadcast_to(np.asarray(nu, np.float64), (conn.shape[0],))
        for e in range(conn.shape[0]):
            d = data[e]
            d.E, d.nu, d.thick, d.tOffset = float(E_arr[e]), float(nu_arr[e]), float(thick[e]), tOffset
            if ref_axis is not None:
                d.refAxis[0], d.refAxis[1], d.refAxis[2] = ref_axis
                d.has_ref_axis = 1
        desc = L.gf_mesh_desc()
        desc.num_nodes = xpts.shape[0]
        desc.num_elements = conn.shape[0]
        self._conn, self._xpts, self._bcs, self._data = conn, xpts, bcs, data
        desc.conn = conn.ctypes.data_as(C.POINTER(C.c_int32))
        desc.xpts = xpts.ctypes.data_as(C.POINTER(C.c_double))
        desc.bcs = bcs.ctypes.data_as(C.POINTER(C.c_int32))
        desc.num_bcs = bcs.size
        desc.data = data
        desc.ordering = {"natural": L.GF_ORDER_NATURAL, "rcm": L.GF_ORDER_RCM,
                         "qorder": L.GF_ORDER_QORDER}[ordering]
        desc.rcm_root = rcm_root
        desc.qorder_p = qorder_p
        desc.qorder_seed = qorder_seed
        h = C.c_void_p()
        torch.cuda.init()
        check(L.lib().gf_assembler_create(C.byref(desc), C.byref(h)), "gf_assembler_create")
        self.h = h
        self.bcs = bcs

    @classmethod
    def createFromBDF(cls, path, E=70e9, nu=0.3, thick=0.005, ordering="natural", **kw):
        """createFromBDF (include/assembler.h:92-115): the mesh of a NASTRAN
        bulk-data file (read_bdf) with one material for every element, as
        the reference's single `Data` argument; `thick` may also be a dict
        from property id (PID) to thickness."""
        m = read_bdf(path)
        if isinstance(thick, dict):
            t = np.array([thick[int(c)] for c in m["component"]], np.float64)
        else:
            t = thick
        return cls(m["conn"], m["xpts"], m["bcs"], t, E, nu, ordering=ordering, **kw)

    @classmethod
    def from_mesh(cls, mesh, ordering="natural", **kw):
        return cls(mesh.conn, mesh.xpts, mesh.bcs, mesh.thick, mesh.E, mesh.nu,
                   ordering=ordering, **kw)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and L._LIB is not None:
            L.lib().gf_assembler_destroy(h)
            self.h = None

    # reference getters (include/assembler.h:117-118, :307-310)
    def get_num_nodes(self):
        return L.lib().gf_assembler_num_nodes(self.h)

    def get_num_elements(self):
        return L.lib().gf_assembler_num_elements(self.h)

    def get_num_vars(self):
        return L.lib().gf_assembler_num_vars(self.h)

    def get_nnzb(self):
        return L.lib().gf_assembler_nnzb(self.h)

    def getBsrData(self):
        n, nnz = self.get_num_nodes(), self.get_nnzb()
        rowp = np.zeros(n + 1, np.int32)
        cols = np.zeros(nnz, np.int32)
        perm = np.zeros(n, np.int32)
        emap = np.zeros(16 * self.get_num_elements(), np.int32)
        check(L.lib().gf_assembler_get_pattern(self.h, _ip(rowp), _ip(cols), _ip(perm),
                                               _ip(emap)), "get_pattern")
        return {"rowPtr": rowp, "colPtr": cols, "perm": perm, "elemIndMap": emap,
                "nnzb": nnz, "nnodes": n}

    def getSchedule(self):
        ne = self.get_num_elements()
        ec, cc_dummy = np.zeros(ne, np.int32), None
        elem_chunk = np.zeros(ne, np.int32)
        elem_color = np.zeros(ne, np.int32)
        ft = np.zeros(ne, np.uint32)
        ncc, nch = C.c_int32(), C.c_int32()
        check(L.lib().gf_assembler_get_schedule(self.h, _ip(elem_chunk), None, _ip(elem_color),
                                                ft.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                C.byref(ncc), C.byref(nch)), "get_schedule")
        chunk_color = np.zeros(nch.value, np.int32)
        check(L.lib().gf_assembler_get_schedule(self.h, None, _ip(chunk_color), None, None,
                                                None, None), "get_schedule")
        return {"elem_chunk": elem_chunk, "chunk_color": chunk_color, "elem_color": elem_color,
                "first_touch": ft, "num_chunk_colors": ncc.value, "num_chunks": nch.value}

    def createVarsVec(self, data=None):
        if data is None:
            return DeviceVec(self.get_num_vars())
        return DeviceVec(torch.as_tensor(np.asarray(data, np.float64)).cuda().contiguous())

    def set_variables(self, vec: DeviceVec):
        check(L.lib().gf_set_variables(self.h, vec.getPtr(), _stream()), "set_variables")

    def set_thickness(self, thick: torch.Tensor):
        """Per-element thickness (natural element order) on the device."""
        check(L.lib().gf_assembler_set_thickness(self.h, _ptr(thick), _stream()), "set_thickness")

    def add_residual(self, res: DeviceVec, add=False, fuse_bcs=False, atomic=False):
        flags = ((L.GF_ASSEMBLE_ADD if add else 0) | (L.GF_ASSEMBLE_FUSE_BCS if fuse_bcs else 0)
                 | (L.GF_ASSEMBLE_ATOMIC if atomic else 0))
        check(L.lib().gf_add_residual(self.h, res.getPtr(), flags, _stream()), "add_residual")

    def add_jacobian(self, res, mat, add=False, fuse_bcs=False, atomic=None):
        """K (and R into `res`) of add_jacobian (include/assembler.h:267). atomic:
        one launch scattering with FP64 atomics instead of the coloured,
        bitwise-reproducible schedule (None: the choice of tune_scatter, else
        coloured)."""
        if atomic is None:
            atomic = getattr(self, "scatter_atomic", False)
        flags = ((L.GF_ASSEMBLE_ADD if add else 0) | (L.GF_ASSEMBLE_FUSE_BCS if fuse_bcs else 0)
                 | (L.GF_ASSEMBLE_ATOMIC if atomic else 0))
        rp = None if res is None else res.getPtr()
        check(L.lib().gf_add_jacobian(self.h, rp, mat.h, flags, _stream()), "add_jacobian")

    def setup_info(self):
        """gf_assembler_setup_info: whether the node pattern and the
        elemIndMap were computed on the GPU."""
        p, m = C.c_int32(), C.c_int32()
        check(L.lib().gf_assembler_setup_info(self.h, C.byref(p), C.byref(m)), "setup_info")
        return {"pattern_on_gpu": bool(p.value), "elem_map_on_gpu": bool(m.value)}

    def tune_scatter(self, mat, reps=5):
        """Times the Jacobian with the coloured and the atomic scatter on
        `mat` and keeps the faster for add_jacobian(atomic=None); returns the
        two times (ms). On a 400x200 plate the atomic one wins (0.62 vs
        0.71 ms: one launch instead of one per colour)."""
        def timed(atomic):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            self.add_jacobian(None, mat, fuse_bcs=True, atomic=atomic)
            e0.record()
            for _ in range(reps):
                self.add_jacobian(None, mat, fuse_bcs=True, atomic=atomic)
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        t = {"coloured": timed(False), "atomic": timed(True)}
        self.scatter_atomic = t["atomic"] < t["coloured"]
        return t

    def add_energy(self):
        out = C.c_double()
        check(L.lib().gf_add_energy(self.h, C.byref(out), _stream()), "add_energy")
        return out.value

    def apply_bcs(self, obj):
        if isinstance(obj, BsrMat):
            check(L.lib().gf_apply_bcs_mat(self.h, obj.h, _stream()), "apply_bcs(mat)")
        else:
            check(L.lib().gf_apply_bcs_vec(self.h, obj.getPtr(), _stream()), "apply_bcs(vec)")


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def order_nodes(conn, num_nodes, ordering="rcm", rcm_root=0, qorder_p=1.0, qorder_seed=0):
    """gf_order_nodes: the solver ordering perm[natural node] = row that an
    assembler of this connectivity would use (host only)."""
    conn = np.ascontiguousarray(conn, np.int32).reshape(-1, 4)
    desc = L.gf_mesh_desc()
    desc.num_nodes = num_nodes
    desc.num_elements = conn.shape[0]
    desc.conn = conn.ctypes.data_as(C.POINTER(C.c_int32))
    desc.ordering = {"natural": L.GF_ORDER_NATURAL, "rcm": L.GF_ORDER_RCM,
                     "qorder": L.GF_ORDER_QORDER}[ordering]
    desc.rcm_root = rcm_root
    desc.qorder_p = qorder_p
    desc.qorder_seed = qorder_seed
    perm = np.zeros(num_nodes, np.int32)
    check(L.lib().gf_order_nodes(C.byref(desc), _ip(perm)), "gf_order_nodes")
    return perm


def read_bdf(path):
    """gf_bdf_read: conn (4 per element, tensor order), xpts, bcs (natural
    DOF indices) and component (property id per element) of a NASTRAN
    bulk-data file, as numpy arrays."""
    mp = C.POINTER(L.gf_bdf_mesh)()
    check(L.lib().gf_bdf_read(os.fsencode(path), C.byref(mp)), "gf_bdf_read")
    try:
        m = mp.contents
        ne, nn, nb = m.num_elements, m.num_nodes, m.num_bcs
        out = {"conn": np.ctypeslib.as_array(m.conn, (max(4 * ne, 1),))[:4 * ne].reshape(ne, 4).copy(),
               "xpts": np.ctypeslib.as_array(m.xpts, (max(3 * nn, 1),))[:3 * nn].reshape(nn, 3).copy(),
               "bcs": (np.ctypeslib.as_array(m.bcs, (nb,)).copy() if nb else np.zeros(0, np.int32)),
               "component": np.ctypeslib.as_array(m.component, (max(ne, 1),))[:ne].copy()}
    finally:
        L.lib().gf_bdf_free(mp)
    return out


class BsrMat:
    """BsrMat<DeviceVec<double>> (include/linalg/bsr_mat.h:9-352)."""

    def __init__(self, assembler: ElementAssembler):
        self.assembler = assembler
        h = C.c_void_p()
        check(L.lib().gf_bsr_create(assembler.h, C.byref(h)), "gf_bsr_create")
        self.h = h
        self.nnzb = assembler.get_nnzb()

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and L._LIB is not None:
            L.lib().gf_bsr_destroy(h)
            self.h = None

    def getPtr(self):
        return L.lib().gf_bsr_values(self.h)

    def zeroValues(self):
        check(L.lib().gf_bsr_zero(self.h, _stream()), "zeroValues")

    def values_host(self):
        torch.cuda.synchronize()
        out = np.zeros(36 * self.nnzb)
        import ctypes
        ctypes_ptr = self.getPtr()
        t = torch.empty(36 * self.nnzb, dtype=torch.float64, device="cuda")
        # copy through cudaMemcpy via torch: wrap raw pointer
        _copy_dev_to_tensor(ctypes_ptr, t)
        out[:] = t.cpu().numpy()
        return out

    def spmv(self, x: torch.Tensor, y: torch.Tensor, alpha=1.0, beta=0.0):
        check(L.lib().gf_bsr_spmv(self.h, alpha, _ptr(x), beta, _ptr(y), _stream()), "spmv")


def _copy_dev_to_tensor(ptr, t):
    import ctypes
    cudart = _cudart()
    cudart.cudaMemcpy(C.c_void_p(t.data_ptr()), C.c_void_p(ptr),
                      C.c_size_t(t.numel() * t.element_size()), 3)
    torch.cuda.synchronize()


_CUDART = None


def _cudart():
    global _CUDART
    if _CUDART is None:
        import glob
        import os
        cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "lib", "libcudart*.so*"))
        cands += ["libcudart.so", "/usr/local/cuda/lib64/libcudart.so"]
        for c in cands:
            try:
                _CUDART = C.CDLL(c)
                break
            except OSError:
                continue
    return _CUDART


def createBsrMat(assembler):
    return BsrMat(assembler)


class ILUk_Preconditioner:
    """ILUk_Preconditioner (include/linalg/precond.h:5-55) with computeILUk's
    symbolic fill (include/linalg/bsr_utils.h:678-807)."""

    def __init__(self, assembler: ElementAssembler, fill_level=0, precision="fp64",
                 sweep="auto"):
        """sweep: "auto", "dataflow" or "level" (gf_precond_create_ex)."""
        self.assembler = assembler
        h = C.c_void_p()
        prec = {"fp64": L.GF_PREC_FP64, "fp32": L.GF_PREC_FP32}[precision]
        kind = {"auto": L.GF_SWEEP_AUTO, "dataflow": L.GF_SWEEP_DATAFLOW,
                "level": L.GF_SWEEP_LEVEL}[sweep]
        check(L.lib().gf_precond_create_ex(assembler.h, fill_level, prec, kind, C.byref(h)),
              "gf_precond_create")
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and L._LIB is not None:
            L.lib().gf_precond_destroy(h)
            self.h = None

    def factor(self, mat: BsrMat):
        check(L.lib().gf_precond_factor(self.h, mat.h, _stream()), "precond_factor")

    def apply(self, r: torch.Tensor, z: torch.Tensor):
        check(L.lib().gf_precond_apply(self.h, _ptr(r), _ptr(z), _stream()), "precond_apply")

    def info(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(L.lib().gf_precond_info(self.h, C.byref(a), C.byref(b), C.byref(c)), "info")
        return {"nnzb": a.value, "levels_L": b.value, "levels_U": c.value}

    def sweeps(self):
        """Sweep kernel of the L and U triangles ("dataflow" / "level") and the
        dataflow result rings' slots."""
        v = [C.c_int32() for _ in range(4)]
        check(L.lib().gf_precond_sweeps(self.h, *[C.byref(x) for x in v]), "sweeps")
        name = {L.GF_SWEEP_DATAFLOW: "dataflow", L.GF_SWEEP_LEVEL: "level"}
        return {"L": name[v[0].value], "U": name[v[1].value], "ring_L": v[2].value,
                "ring_U": v[3].value}

    def layout(self):
        v = [C.c_int32() for _ in range(5)]
        check(L.lib().gf_precond_layout(self.h, *[C.byref(x) for x in v]), "layout")
        return {"nsplit_L": v[0].value, "nsplit_U": v[1].value, "fac_ctas": v[2].value,
                "chunks_L": v[3].value, "chunks_U": v[4].value}

    def setup_info(self):
        """gf_precond_setup_info: whether the ILU(k) pattern was computed on
        the GPU, and the host wall times (ms) of the pattern and the setup."""
        g, sm, tm = C.c_int32(), C.c_double(), C.c_double()
        check(L.lib().gf_precond_setup_info(self.h, C.byref(g), C.byref(sm), C.byref(tm)),
              "setup_info")
        return {"symbolic_on_gpu": bool(g.value), "symbolic_ms": sm.value, "setup_ms": tm.value}

    def status(self):
        """gf_precond_status: reads and clears the device-side status flags."""
        return L.lib().gf_precond_status(self.h, _stream())

    def get(self):
        inf = self.info()
        n = self.assembler.get_num_nodes()
        rowp = np.zeros(n + 1, np.int32)
        cols = np.zeros(inf["nnzb"], np.int32)
        vals = np.zeros(36 * inf["nnzb"])
        check(L.lib().gf_precond_get(self.h, _ip(rowp), _ip(cols),
                                     vals.ctypes.data_as(C.POINTER(C.c_double))), "get")
        return rowp, cols, vals


class SolveOptions(L.gf_solve_opts):
    def __init__(self, **kw):
        super().__init__()
        L.lib().gf_solve_opts_default(C.byref(self))
        for k, v in kw.items():
            setattr(self, k, v)


def gmres_solve(assembler, mat, precond, b: torch.Tensor, x: torch.Tensor, opts=None,
                raise_on_fail=True):
    """ILU-preconditioned GMRES of examples/iterative/gmres.cu:468-771."""
    opts = opts or SolveOptions()
    stats = L.gf_solve_stats()
    st = L.lib().gf_gmres_solve(assembler.h, mat.h, precond.h, _ptr(b), _ptr(x), C.byref(opts),
                                C.byref(stats), _stream())
    if raise_on_fail and st not in (L.GF_OK, L.GF_NOT_CONVERGED):
        check(st, "gmres_solve")
    return st, {"iterations": stats.iterations, "restarts": stats.restarts,
                "refinements": stats.refinements, "status": stats.status,
                "rel_residual": stats.rel_residual, "time_ms": stats.time_ms}


def direct_solve(assembler, mat, b: torch.Tensor, x: torch.Tensor, raise_on_fail=True):
    """Complete block LU solve of CUSPARSE::direct_LU_solve_old
    (include/linalg/solvers/cusparse.h:16-192) through gf_direct_solve: the
    full-fill factor on the ILU kernels, applied with GMRES refinement to the
    FP64 residual floor."""
    stats = L.gf_solve_stats()
    st = L.lib().gf_direct_solve(assembler.h, mat.h, _ptr(b), _ptr(x), C.byref(stats), _stream())
    if raise_on_fail:
        check(st, "direct_solve")
    return st, {"iterations": stats.iterations, "status": stats.status,
                "rel_residual": stats.rel_residual, "time_ms": stats.time_ms}


direct_LU_solve_old = direct_solve
