"""GPU parity of the assembly path against the CPU oracle.

Residual and Jacobian entries within 1e-12 relative (absolute floor
1e-12 * max|K|), pattern / elemIndMap / schedule bit-exact, BCs exact.
"""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _close(a, b, tol=RTOL):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err <= tol, f"max rel err {err:.3e} > {tol:.1e}"
    return err


def one_element_mesh():
    """tests/shell_res/local_utils.h:5-38 (xpts formula) with vars of res.cu:33-36."""
    xpts = np.array([1.0345452 + 2.23123432 * i + 0.323 * i * i for i in range(12)]).reshape(4, 3)
    conn = np.array([[0, 1, 2, 3]], np.int32)
    m = M.ShellMesh(conn, xpts, np.array([0.005]), np.zeros(0, np.int32), np.zeros(24),
                    70e9, 0.3, "one_element")
    u = np.array([(1.4543 + 6.4323 * i) * 1e-6 for i in range(24)])
    return m, u


def meshes():
    m1 = M.plate_config1()
    m2 = M.plate_config2(24, 12)
    bx = M.box(nx=18, ny=6, nz=4, nribs=4)
    return [("plate10", m1, "natural"), ("plate24x12_rcm", m2, "rcm"), ("box", bx, "rcm")]


def _assemble_gpu(mesh, ordering, u=None, fuse=False):
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, createBsrMat
    A = ElementAssembler.from_mesh(mesh, ordering=ordering)
    if u is not None:
        A.set_variables(A.createVarsVec(u))
    K = createBsrMat(A)
    res = A.createVarsVec()
    A.add_jacobian(res, K, fuse_bcs=fuse)
    torch.cuda.synchronize()
    return A, K, res


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_jacobian_and_residual_match_oracle(oracle, idx):
    name, mesh, ordering = meshes()[idx]
    rng = np.random.default_rng(7)
    u = rng.standard_normal(mesh.num_dof) * 1e-4
    A, K, res = _assemble_gpu(mesh, ordering, u)
    bd = A.getBsrData()
    rowp, cols, vals, r_or, perm = oracle.assemble_jacobian(mesh, u, perm=bd["perm"])
    np.testing.assert_array_equal(bd["rowPtr"], rowp)
    np.testing.assert_array_equal(bd["colPtr"], cols)
    np.testing.assert_array_equal(bd["elemIndMap"], oracle.elem_ind_map(mesh.conn, rowp, cols,
                                                                        perm))
    _close(K.values_host(), vals)
    _close(res.t.cpu().numpy(), r_or, 1e-11)


def test_one_element_fixture(oracle):
    mesh, u = one_element_mesh()
    A, K, res = _assemble_gpu(mesh, "natural", u)
    rowp, cols, vals, r_or, perm = oracle.assemble_jacobian(mesh, u)
    _close(K.values_host(), vals)
    _close(res.t.cpu().numpy(), r_or, 1e-11)
    # residual-only kernel and energy
    res2 = A.createVarsVec()
    A.add_residual(res2)
    _close(res2.t.cpu().numpy(), oracle.assemble_residual(mesh, u), 1e-11)
    d = oracle.make_data(70e9, 0.3, 0.005)
    U = A.add_energy()
    assert abs(U - oracle.element_energy(mesh.xpts, u, d)) <= 1e-12 * abs(U)


def test_residual_kernel_matches_oracle(oracle):
    mesh = M.plate_config2(24, 12)
    u = np.random.default_rng(3).standard_normal(mesh.num_dof) * 1e-3
    from gpu_fem_b200.assembler import ElementAssembler
    A = ElementAssembler.from_mesh(mesh, ordering="rcm")
    A.set_variables(A.createVarsVec(u))
    r = A.createVarsVec()
    A.add_residual(r)
    _close(r.t.cpu().numpy(), oracle.assemble_residual(mesh, u), 1e-11)
    # additive mode doubles it
    A.add_residual(r, add=True)
    _close(r.t.cpu().numpy(), 2 * oracle.assemble_residual(mesh, u), 1e-11)


def test_bcs_separate_and_fused_match_oracle(oracle):
    mesh = M.plate_config2(24, 12)
    u = np.random.default_rng(5).standard_normal(mesh.num_dof) * 1e-4
    A, K, res = _assemble_gpu(mesh, "rcm", u)
    A.apply_bcs(K)
    A.apply_bcs(res)
    bd = A.getBsrData()
    rowp, cols, vals, r_or, perm = oracle.assemble_jacobian(mesh, u, perm=bd["perm"])
    oracle.apply_bcs_mat(rowp, cols, vals, perm, mesh.bcs)
    r_or[mesh.bcs] = 0.0
    _close(K.values_host(), vals)
    _close(res.t.cpu().numpy(), r_or, 1e-11)
    A2, K2, res2 = _assemble_gpu(mesh, "rcm", u, fuse=True)
    _close(K2.values_host(), vals)
    _close(res2.t.cpu().numpy(), r_or, 1e-11)


def test_schedule_bit_exact_and_deterministic(oracle):
    from oracle.schedule import schedule
    mesh = M.plate_config2(24, 12)
    A, K, res = _assemble_gpu(mesh, "rcm")
    s = A.getSchedule()
    ref = schedule(mesh.conn, mesh.num_nodes, A.getBsrData()["elemIndMap"], chunk_size=8)
    for k in ("elem_chunk", "chunk_color", "elem_color", "first_touch"):
        np.testing.assert_array_equal(s[k], ref[k], err_msg=k)
    assert s["num_chunk_colors"] == ref["num_chunk_colors"]
    v1 = K.values_host()
    A.add_jacobian(res, K)
    v2 = K.values_host()
    assert np.array_equal(v1.view(np.uint64), v2.view(np.uint64))


def test_rcm_matches_oracle(oracle):
    mesh = M.plate_config2(30, 15)
    from gpu_fem_b200.assembler import ElementAssembler
    A = ElementAssembler.from_mesh(mesh, ordering="rcm")
    rowp0, cols0 = oracle.bsr_pattern(mesh.conn, mesh.num_nodes)
    np.testing.assert_array_equal(A.getBsrData()["perm"], oracle.rcm(rowp0, cols0, 0, 1))


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_atomic_scatter_matches_coloured(idx):
    """GF_ASSEMBLE_ATOMIC (one launch, FP64 atomics; the reference's scatter)
    against the coloured schedule: K and R within 1e-13 of max |K| / |R|,
    with and without fused BCs, and the diagonal 1.0 of each constrained DOF
    added exactly once."""
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, createBsrMat
    name, mesh, ordering = meshes()[idx]
    A = ElementAssembler.from_mesh(mesh, ordering=ordering)
    u = np.random.default_rng(5).standard_normal(mesh.num_dof) * 1e-3
    A.set_variables(A.createVarsVec(u))
    for fuse in (False, True):
        Kc, Ka = createBsrMat(A), createBsrMat(A)
        rc, ra = A.createVarsVec(), A.createVarsVec()
        A.add_jacobian(rc, Kc, fuse_bcs=fuse)
        A.add_jacobian(ra, Ka, fuse_bcs=fuse, atomic=True)
        torch.cuda.synchronize()
        _close(Ka.values_host(), Kc.values_host(), 1e-13)
        _close(ra.t.cpu().numpy(), rc.t.cpu().numpy(), 1e-13)
    r1, r2 = A.createVarsVec(), A.createVarsVec()
    A.add_residual(r1)
    A.add_residual(r2, atomic=True)
    torch.cuda.synchronize()
    _close(r2.t.cpu().numpy(), r1.t.cpu().numpy(), 1e-13)


def test_batched_assembly_coloured_bitwise_and_atomic_close():
    """gf_batch_assemble runs each colour of all problems in one launch: K is
    bitwise the one gf_add_jacobian gives per problem; with the atomic
    scatter (one launch) within 1e-13 of max |K|."""
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner, createBsrMat
    from gpu_fem_b200.batch import Batch
    ms = [M.plate_config2(24, 12), M.box(nx=18, ny=6, nz=4, nribs=4), M.plate_config1()]
    asms = [ElementAssembler.from_mesh(m, ordering="rcm") for m in ms]
    mats = [createBsrMat(a) for a in asms]
    pcs = [ILUk_Preconditioner(a, fill_level=1) for a in asms]
    ref = []
    for a in asms:
        K = createBsrMat(a)
        a.add_jacobian(None, K, fuse_bcs=True)
        ref.append(K)
    torch.cuda.synchronize()
    bt = Batch(asms, mats, pcs)
    bt.assemble()
    torch.cuda.synchronize()
    for K, R in zip(mats, ref):
        assert np.array_equal(K.values_host().view(np.uint64), R.values_host().view(np.uint64))
    bt.set_scatter(True)
    bt.assemble()
    torch.cuda.synchronize()
    for K, R in zip(mats, ref):
        _close(K.values_host(), R.values_host(), 1e-13)
