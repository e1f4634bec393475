"""GPU parity of SpMV, block ILU(k), triangular solves and GMRES."""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _system(mesh, ordering, oracle):
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, createBsrMat
    A = ElementAssembler.from_mesh(mesh, ordering=ordering)
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    torch.cuda.synchronize()
    bd = A.getBsrData()
    rowp, cols, vals, _, perm = oracle.assemble_jacobian(mesh, perm=bd["perm"])
    oracle.apply_bcs_mat(rowp, cols, vals, perm, mesh.bcs)
    return A, K, rowp, cols, vals, perm


def _to_solver(v, perm):
    out = np.zeros_like(v)
    out.reshape(-1, 6)[perm] = v.reshape(-1, 6)
    return out


def test_spmv_matches_oracle(oracle):
    import torch
    mesh = M.plate_config2(24, 12)
    A, K, rowp, cols, vals, perm = _system(mesh, "rcm", oracle)
    x = np.random.default_rng(1).standard_normal(mesh.num_dof)
    y_ref = oracle.spmv(rowp, cols, vals, x)
    xt = torch.tensor(x, device="cuda")
    yt = torch.zeros_like(xt)
    K.spmv(xt, yt)
    y = yt.cpu().numpy()
    assert np.abs(y - y_ref).max() <= 1e-13 * np.abs(y_ref).max()


@pytest.mark.parametrize("fill", [0, 2])
def test_ilu_factor_and_apply_match_oracle(oracle, fill):
    import torch
    from gpu_fem_b200.assembler import ILUk_Preconditioner
    mesh = M.plate_config2(24, 12)
    A, K, rowp, cols, vals, perm = _system(mesh, "rcm", oracle)
    P = ILUk_Preconditioner(A, fill_level=fill)
    P.factor(K)
    torch.cuda.synchronize()
    r2, c2, lu_gpu = P.get()
    if fill:
        rk, ck = oracle.iluk_pattern(rowp, cols, fill)
        np.testing.assert_array_equal(r2, rk)
        np.testing.assert_array_equal(c2, ck)
        vals_k = oracle.scatter_to_pattern(rowp, cols, vals, rk, ck)
    else:
        np.testing.assert_array_equal(r2, rowp)
        np.testing.assert_array_equal(c2, cols)
        vals_k = vals
    st, lu_ref = oracle.ilu0(r2, c2, vals_k)
    assert st == 0
    # Block ILU on these shells is numerically unstable (factor growth
    # ~1e13), so two correct factorizations that round in a different order
    # differ entrywise far above machine precision. Parity is measured by what
    # ILU(k) defines: (L U)_ij = A_ij on the pattern (backward error), for the
    # GPU factors (diagonal blocks hold U_ii^{-1}) and for the oracle's, plus
    # bitwise run-to-run equality.
    n = len(r2) - 1
    G = lu_gpu.reshape(-1, 6, 6).copy()
    for i in range(n):
        for jp in range(r2[i], r2[i + 1]):
            if c2[jp] == i:
                G[jp] = np.linalg.inv(G[jp])
    A_d = oracle.bsr_to_dense(r2, c2, vals_k)
    mask = oracle.bsr_to_dense(r2, c2, np.ones(36 * len(c2))) != 0

    def backward(F):
        """max |(L U - A)_ij| over the pattern / max |A| for block factors F."""
        N = 6 * n
        Lm, Um = np.eye(N), np.zeros((N, N))
        for i in range(n):
            for jp in range(r2[i], r2[i + 1]):
                j = c2[jp]
                tgt = Lm if j < i else Um
                tgt[6 * i:6 * i + 6, 6 * j:6 * j + 6] = F[jp]
        LU = Lm @ Um
        return np.abs((LU - A_d)[mask]).max() / np.abs(A_d).max(), Lm, Um

    eg, Lg, Ug = backward(G)
    eo, _, _ = backward(lu_ref.reshape(-1, 6, 6))
    assert eo <= 1e-10, eo
    assert eg <= 1e-10, eg
    P.factor(K)
    torch.cuda.synchronize()
    _, _, lu_again = P.get()
    assert np.array_equal(lu_again.view(np.uint64), lu_gpu.view(np.uint64))
    # the apply solves L U z = r with the GPU factors (triangular solves are
    # backward stable)
    r = np.random.default_rng(2).standard_normal(mesh.num_dof)
    rt = torch.tensor(r, device="cuda")
    zt = torch.zeros_like(rt)
    P.apply(rt, zt)
    z = zt.cpu().numpy()
    res = Lg @ (Ug @ z) - r
    scale = np.abs(Lg).max() * np.abs(Ug).max() * np.abs(z).max() * len(z)
    assert np.abs(res).max() <= 1e-13 * scale


@pytest.mark.parametrize("side", [0, 1])
def test_gmres_config1_matches_dense_solve(oracle, side):
    import torch
    from gpu_fem_b200.assembler import ILUk_Preconditioner, SolveOptions, gmres_solve
    mesh = M.plate_config1()
    A, K, rowp, cols, vals, perm = _system(mesh, "natural", oracle)
    x_dense = oracle.dense_solve(oracle.bsr_to_dense(rowp, cols, vals), mesh.loads)
    P = ILUk_Preconditioner(A, fill_level=0)
    P.factor(K)
    b = torch.tensor(mesh.loads, device="cuda")
    x = torch.zeros_like(b)
    st, stats = gmres_solve(A, K, P, b, x, SolveOptions(restart=300, max_iters=3000, rtol=1e-10,
                                                        side=side))
    assert stats["rel_residual"] <= 1e-9, stats
    err = np.linalg.norm(x.cpu().numpy() - x_dense) / np.linalg.norm(x_dense)
    assert err <= 1e-8, (err, stats)


def test_mixed_precision_refinement_reaches_fp64_tolerance(oracle):
    import torch
    from gpu_fem_b200.assembler import ILUk_Preconditioner, SolveOptions, gmres_solve
    mesh = M.plate(32, 32, 1.0, 1.0, lambda x, y: 0.005 + 0 * x, "all_edges",
                   lambda q: 1e3 + 0 * q[:, 0])
    A, K, rowp, cols, vals, perm = _system(mesh, "rcm", oracle)
    x_dense = oracle.dense_solve(oracle.bsr_to_dense(rowp, cols, vals),
                                 _to_solver(mesh.loads, perm))
    x_dense = x_dense.reshape(-1, 6)[perm].ravel()
    b = torch.tensor(mesh.loads, device="cuda")
    # block ILU(k) convergence is not monotonic in k on thin shells: on this
    # plate the oracle's own ILU(2) stalls in right-preconditioned GMRES(200)
    # while ILU(1) and ILU(3) converge, so ILU(3) is used
    for mixed, prec in ((0, "fp64"), (1, "fp32")):
        P = ILUk_Preconditioner(A, fill_level=3, precision=prec)
        P.factor(K)
        x = torch.zeros_like(b)
        # solved to 1e-10 (this plate's FP64 rounding floor eps || |A| |x| ||
        # / ||b|| is 5e-11)
        # so that the displacement gate, 1e-8 relative to the dense FP64
        # solve, does not depend on where the iteration stopped
        st, stats = gmres_solve(A, K, P, b, x, SolveOptions(restart=200, max_iters=4000,
                                                            rtol=1e-10, mixed=mixed, side=1,
                                                            inner_rtol=1e-3))
        assert stats["rel_residual"] <= 1e-10, (mixed, stats)
        err = np.linalg.norm(x.cpu().numpy() - x_dense) / np.linalg.norm(x_dense)
        assert err <= 1e-8, (mixed, err, stats)


def test_precond_apply_accepts_8_byte_aligned_vectors():
    """The sweeps move 6-double rows as 16-byte pieces when the vectors allow
    and as 8-byte pieces otherwise; both give the same z bit for bit."""
    import torch
    from gpu_fem_b200.assembler import ILUk_Preconditioner
    mesh = M.plate_config2(24, 12)
    from gpu_fem_b200.assembler import ElementAssembler, createBsrMat
    A = ElementAssembler.from_mesh(mesh, ordering="rcm")
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    for prec in ("fp64", "fp32"):
        P = ILUk_Preconditioner(A, fill_level=2, precision=prec)
        P.factor(K)
        n = mesh.num_dof
        r = torch.tensor(np.random.default_rng(5).standard_normal(n), device="cuda")
        z = torch.zeros_like(r)
        P.apply(r, z)
        rb = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
        zb = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
        rb[1:] = r
        P.apply(rb[1:], zb[1:])  # both vectors 8 bytes off a 16-byte boundary
        torch.cuda.synchronize()
        assert np.array_equal(z.cpu().numpy().view(np.uint64), zb[1:].cpu().numpy().view(np.uint64))


def test_status_codes_zero_pivot_and_not_converged():
    """A singular diagonal block is reported as GF_ZERO_PIVOT (no fault), and
    an iteration cap that is too small as GF_NOT_CONVERGED with the achieved
    residual."""
    import torch
    from gpu_fem_b200 import _lib as L
    from gpu_fem_b200.assembler import (ElementAssembler, ILUk_Preconditioner, SolveOptions,
                                        createBsrMat, gmres_solve)
    mesh = M.plate_config2(24, 12)
    A = ElementAssembler.from_mesh(mesh, ordering="rcm")
    K = createBsrMat(A)
    K.zeroValues()  # every block zero: the first pivot block is singular
    P = ILUk_Preconditioner(A, fill_level=0)
    with pytest.raises(L.GpuFemError) as err:
        P.factor(K)
    assert err.value.status == L.GF_ZERO_PIVOT
    A.add_jacobian(None, K, fuse_bcs=True)
    P.factor(K)  # the context is still usable
    b = torch.tensor(mesh.loads, device="cuda")
    x = torch.zeros_like(b)
    st, stats = gmres_solve(A, K, P, b, x, SolveOptions(restart=10, max_iters=3, rtol=1e-12,
                                                        side=1), raise_on_fail=False)
    assert st == L.GF_NOT_CONVERGED
    assert stats["iterations"] <= 3 and stats["rel_residual"] > 1e-12


def test_qordered_ilu_gmres_matches_dense_solve(oracle):
    """The deterministic q-ordering (RCM shuffled within bandwidth-wide windows)
    as the solver ordering: pattern and permutation as the oracle's, the
    ILU(2)-GMRES displacement within 1e-8 of a dense FP64 solve."""
    import torch
    from gpu_fem_b200.assembler import (ElementAssembler, ILUk_Preconditioner, SolveOptions,
                                        createBsrMat, gmres_solve)
    m = M.plate(16, 16, 1.0, 1.0, lambda x, y: 0.006 + 0 * x, "all_edges",
                lambda q: 1e3 + 0 * q[:, 0])
    A = ElementAssembler.from_mesh(m, ordering="qorder", qorder_p=1.0, qorder_seed=42)
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    bd = A.getBsrData()
    rowp0, cols0 = oracle.bsr_pattern(m.conn, m.num_nodes)
    perm = oracle.qorder(rowp0, cols0, oracle.rcm(rowp0, cols0, 0, 1), 1.0, 42)
    np.testing.assert_array_equal(bd["perm"], perm)
    rowp, cols, vals, _, _ = oracle.assemble_jacobian(m, perm=perm)
    oracle.apply_bcs_mat(rowp, cols, vals, perm, m.bcs)
    b = np.zeros(m.num_dof)
    b.reshape(-1, 6)[perm] = m.loads.reshape(-1, 6)
    xd = oracle.dense_solve(oracle.bsr_to_dense(rowp, cols, vals), b).reshape(-1, 6)[perm].ravel()
    P = ILUk_Preconditioner(A, fill_level=2)
    P.factor(K)
    bt = torch.tensor(m.loads, device="cuda")
    x = torch.zeros_like(bt)
    st, stats = gmres_solve(A, K, P, bt, x, SolveOptions(restart=200, max_iters=4000, rtol=1e-10))
    assert stats["rel_residual"] <= 1e-10, stats
    err = np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd)
    assert err <= 1e-8, err
