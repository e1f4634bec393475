"""GPU parity of the large-problem paths of the block ILU factorization and of
the triangular sweeps, the paths the large batched problems run.

Case: 256 x 128 clamped plate, t = 2 mm, natural node ordering, ILU(6):
33,153 block rows and 1,281 levels per triangle, about 26 rows and 405 (L) /
431 (U) blocks per level. The dataflow factorization runs on 128 CTAs whose
warps take rows in level order and wait per step for the rows they read.
The sweeps are checked in both kernels:
- level-synchronous (the default): with FP32 factors both sweeps split
  every chunk over the two CTAs (26 rows a level, more than one CTA's 16
  warps); with FP64 factors a level (~405 blocks) spans two chunks of one
  CTA (a chunk stage holds 208 FP64 blocks), which the chunk model makes
  cheaper than splitting, so near and far x entries cross chunk boundaries.
  A 512 x 128 plate (43 rows, ~670 blocks a level) has FP64 levels split
  over both CTAs and spanning two split chunks each;
- dataflow: every row waits only for the rows it multiplies, through a
  1024-slot result ring that its flow control recycles 32 times per sweep.

Checked, with FP64 and FP32 factor values:
- the layout really is split / multi-CTA (gf_precond_layout);
- the factor's backward error max |(L U - A)_ij| over the ILU pattern is
  within 1e-10 max |A| (sparse block products in the oracle), and two
  factorizations are bitwise equal; ILU(k) is defined by (L U)_ij = A_ij on
  the pattern, and entrywise comparison with another factorization is
  meaningless on these shells (factor growth, see test_gpu_solver);
- the apply z against the oracle's block triangular solves run on the GPU's
  own factor values (rounded to FP32 for FP32 factors), within 1e-12 of
  max |z| (cusparseDbsrsv2_solve semantics, examples/iterative/gmres.cu:522-532);
- the displacement of a GMRES solve to 1e-8 against scipy's SuperLU direct
  solve plus one step of FP64 iterative refinement, within 1e-8 relative;
- two split problems give bitwise the same displacement alone and in one
  batch.
"""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _plate(nx, ny, t=0.002, p=1e3):
    return M.plate(nx, ny, 1.0, ny / nx, lambda x, y: t + 0 * x, "all_edges",
                   lambda q: p + 0 * q[:, 0], name=f"plate_{nx}x{ny}")


@pytest.fixture(scope="module")
def big():
    """256x128 plate: GPU assembler and K, K on host, ILU(6) pattern, A on it."""
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, createBsrMat
    from oracle import pyoracle as po
    mesh = _plate(256, 128)
    A = ElementAssembler.from_mesh(mesh, ordering="natural")
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    torch.cuda.synchronize()
    bd = A.getBsrData()
    rowp, cols = bd["rowPtr"], bd["colPtr"]
    vals = K.values_host()
    rk, ck = po.iluk_pattern(rowp, cols, 6)
    Ak = po.scatter_to_pattern(rowp, cols, vals, rk, ck)
    return {"mesh": mesh, "A": A, "K": K, "rowp": rowp, "cols": cols, "vals": vals, "rk": rk,
            "ck": ck, "Ak": Ak}


def _layout(P):
    import ctypes as C
    from gpu_fem_b200 import _lib as L
    v = [C.c_int32() for _ in range(5)]
    L.check(L.lib().gf_precond_layout(P.h, *[C.byref(x) for x in v]), "layout")
    return [x.value for x in v]


@pytest.mark.parametrize("sweep", ["level", "dataflow"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_split_factor_and_apply_match_oracle(big, precision, sweep):
    import torch
    from gpu_fem_b200.assembler import ILUk_Preconditioner
    from oracle import pyoracle as po
    P = ILUk_Preconditioner(big["A"], fill_level=6, precision=precision, sweep=sweep)
    nsL, nsU, fsplit, chL, chU = _layout(P)
    inf = P.info()
    assert fsplit == 128
    kinds = P.sweeps()
    assert kinds["L"] == kinds["U"] == sweep, kinds
    if sweep == "level":
        if precision == "fp32":
            assert (nsL, nsU) == (2, 2), (nsL, nsU)
        else:
            # one CTA, levels larger than one chunk: more chunks than levels
            assert (nsL, nsU) == (1, 1), (nsL, nsU)
            assert chL > inf["levels_L"] and chU > inf["levels_U"], (chL, chU, inf)
    else:
        assert kinds["ring_L"] == kinds["ring_U"] == 1024, kinds
    P.factor(big["K"])
    torch.cuda.synchronize()
    r2, c2, lu = P.get()
    np.testing.assert_array_equal(r2, big["rk"])
    np.testing.assert_array_equal(c2, big["ck"])
    err, amax = po.ilu_backward_error(r2, c2, lu, big["Ak"], dinv=True)
    assert err <= 1e-10 * amax, (err, amax)
    P.factor(big["K"])
    torch.cuda.synchronize()
    _, _, lu2 = P.get()
    assert np.array_equal(lu2.view(np.uint64), lu.view(np.uint64))
    # the sweeps on the GPU's own factor values (the FP32 streams hold them
    # rounded to nearest FP32; products accumulate in FP64 on both sides)
    lu_used = lu.astype(np.float32).astype(np.float64) if precision == "fp32" else lu
    rng = np.random.default_rng(11)
    for call in range(2):
        r = rng.standard_normal(big["mesh"].num_dof)
        rt = torch.tensor(r, device="cuda")
        zt = torch.zeros_like(rt)
        P.apply(rt, zt)
        z = zt.cpu().numpy()
        z_ref = po.ilu_apply_dinv(r2, c2, lu_used, r)
        scale = np.abs(z_ref).max()
        assert np.abs(z - z_ref).max() <= 1e-12 * scale, (call, np.abs(z - z_ref).max() / scale)


def test_split_multichunk_levels_match_oracle():
    """512 x 128 plate, natural order, ILU(6), FP64 factors: every level is
    split over the two CTAs and spans two split chunks; the factor's
    backward error and the apply against the oracle's triangular solves."""
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner, createBsrMat
    from oracle import pyoracle as po
    mesh = _plate(512, 128)
    A = ElementAssembler.from_mesh(mesh, ordering="natural")
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    P = ILUk_Preconditioner(A, fill_level=6, precision="fp64", sweep="level")
    nsL, nsU, _, chL, chU = _layout(P)
    inf = P.info()
    assert (nsL, nsU) == (2, 2), (nsL, nsU)
    assert chL > inf["levels_L"] and chU > inf["levels_U"], (chL, chU, inf)
    P.factor(K)
    torch.cuda.synchronize()
    bd = A.getBsrData()
    rk, ck, lu = P.get()
    Ak = po.scatter_to_pattern(bd["rowPtr"], bd["colPtr"], K.values_host(), rk, ck)
    err, amax = po.ilu_backward_error(rk, ck, lu, Ak, dinv=True)
    assert err <= 1e-10 * amax, (err, amax)
    r = np.random.default_rng(12).standard_normal(mesh.num_dof)
    rt = torch.tensor(r, device="cuda")
    zt = torch.zeros_like(rt)
    P.apply(rt, zt)
    z_ref = po.ilu_apply_dinv(rk, ck, lu, r)
    scale = np.abs(z_ref).max()
    assert np.abs(zt.cpu().numpy() - z_ref).max() <= 1e-12 * scale


def _superlu(mesh, rowp, cols, vals, perm):
    """Direct FP64 solve (SuperLU) plus one step of FP64 iterative refinement,
    in natural node order."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    n = len(rowp) - 1
    S = sp.bsr_matrix((vals.reshape(-1, 6, 6), cols, rowp), shape=(6 * n, 6 * n)).tocsc()
    b = np.zeros(6 * n)
    b.reshape(-1, 6)[perm] = mesh.loads.reshape(-1, 6)
    lu = spl.splu(S)
    x = lu.solve(b)
    x = x + lu.solve(b - S @ x)
    return x.reshape(-1, 6)[perm].ravel()


@pytest.mark.parametrize("sweep", ["level", "dataflow"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_split_solve_matches_direct_solve(big, precision, sweep):
    import torch
    from gpu_fem_b200.assembler import ILUk_Preconditioner, SolveOptions, gmres_solve
    x_ref = big.get("x_ref")
    if x_ref is None:
        x_ref = big["x_ref"] = _superlu(big["mesh"], big["rowp"], big["cols"], big["vals"],
                                        big["A"].getBsrData()["perm"])
    P = ILUk_Preconditioner(big["A"], fill_level=6, precision=precision, sweep=sweep)
    P.factor(big["K"])
    b = torch.tensor(big["mesh"].loads, device="cuda")
    x = torch.zeros_like(b)
    st, stats = gmres_solve(big["A"], big["K"], P, b, x,
                            SolveOptions(restart=100, max_iters=5000, rtol=1e-8, side=1))
    assert stats["rel_residual"] <= 1e-8, stats
    err = np.linalg.norm(x.cpu().numpy() - x_ref) / np.linalg.norm(x_ref)
    assert err <= 1e-8, (precision, err, stats)


def test_split_problems_bitwise_alone_and_in_batch():
    from gpu_fem_b200.assembler import ILUk_Preconditioner
    from gpu_fem_b200.batch import BatchSolver
    meshes = [_plate(200, 100, 0.002, 1e3), _plate(240, 96, 0.003, 1.4e3)]
    bs = BatchSolver(meshes, ordering="natural", fill=6, tune=False)
    for P in bs.P32:
        lay = _layout(P)
        # at least one triangle split over the cluster's two CTAs
        assert max(lay[:2]) == 2 and lay[2] == 128 and P.sweeps()["L"] == "level", lay
    stats = bs.step(True)
    assert all(s["rel_residual"] <= 1e-8 for s in stats), stats
    x_mix = [x.cpu().numpy().copy() for x in bs.xs]
    for i, m in enumerate(meshes):
        alone = BatchSolver([m], ordering="natural", fill=6, tune=False)
        alone.step(True)
        xa = alone.xs[0].cpu().numpy()
        assert np.array_equal(xa.view(np.uint64), x_mix[i].view(np.uint64)), (
            m.name, np.abs(xa - x_mix[i]).max())
