"""Writes the FP64 direct-solve goldens of the scale meshes (test fixtures).

Test infrastructure: run offline on a CPU host, not by the tests. For each
mesh, K is assembled by the CPU oracle in natural node order with the
Dirichlet rows and columns eliminated, and solved with scipy's SuperLU
(symmetric mode: minimum-degree ordering of A + A^T, diagonal pivots; K is
symmetric positive definite) followed by iterative refinement whose
residual b - K x is accumulated in x87 extended precision (64-bit
significand), so that the refinement converges to the correctly rounded
FP64 solution instead of stalling at FP64's residual noise (iterative
refinement with extra-precise residuals). The role of the reference's direct
solve (examples/plate_demo/linear_static.cu:12-73,
CUSPARSE::direct_LU_solve_old) is played by this solve.

Stored per mesh (npz):
  x            displacements (natural order), all DOFs or every `stride`-th
  idx          the DOF indices of x
  xnorm        ||x||_2 over all DOFs
  rel_res      ||b - K x|| / ||b|| of the stored solution (extended precision)
  floor        eps || |K| |x| || / ||b||: the relative residual that rounding
               x to FP64 alone leaves, so no FP64 solution can have a
               smaller one
  fp64_noise   largest relative correction ||dx|| / ||x|| of the last three
               refinement steps when the residual is computed in FP64: how
               far an exactly factored solve moves under FP64 rounding alone
  last_dx      relative size of the last extended-precision correction (the
               stored x is settled to about this)
  k_noise      largest ||x' - x|| / ||x|| over two solves (extended-precision
               refinement) of K' x' = b, where K' is K with every entry
               perturbed by a random relative amount of at most eps: how
               far rounding in an FP64 assembly of K alone moves x, so no
               FP64 assembly and solve can be expected to agree with x
               more closely than this
  mesh         the generator call, for the record

Meshes:
  config2_100x50   the jittered cantilever plate of the scale workload at
                   100 x 50 elements (30,906 DOF), all DOFs
  config2_400x200  the same at its stated size, 400 x 200 (483,606 DOF),
                   every 97th DOF
  box_72x18x6      the stiffened box at a reduced, stated size: 72 x 18 x 6
                   grid (span x chord x depth), 10 ribs, 2 spars, skins 3 mm,
                   webs 6 mm, root clamped, 10 kN tip load; all DOFs
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

EPS = np.finfo(np.float64).eps / 2


def solve(mesh):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    from oracle import pyoracle as po
    rowp, cols, A, _, perm = po.assemble_jacobian(mesh, nthreads=os.cpu_count() or 1)
    po.apply_bcs_mat(rowp, cols, A, perm, mesh.bcs, fast=True)
    n = 6 * mesh.num_nodes
    S = sp.bsr_matrix((A.reshape(-1, 6, 6), cols, rowp), shape=(n, n)).tocsc()
    b = mesh.loads
    lu = spl.splu(S, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                  options=dict(SymmetricMode=True))
    x = lu.solve(b)
    dx = []
    for _ in range(6):  # FP64 residuals: measures the FP64 noise of x
        d = lu.solve(b - S @ x)
        x = x + d
        dx.append(np.linalg.norm(d) / np.linalg.norm(x))
    # extended-precision residuals: r = b - K x with every product and sum in
    # long double, rounded to FP64 once
    Ab = A.reshape(-1, 6, 6).astype(np.longdouble)
    bl = b.astype(np.longdouble)

    def resid(xv, Ab=Ab):
        xb = xv.reshape(-1, 6).astype(np.longdouble)[cols]
        prod = np.einsum("kij,kj->ki", Ab, xb)
        return (bl - np.add.reduceat(prod, rowp[:-1], axis=0).ravel())

    def refine(xv, Ab):
        last = 1.0
        for _ in range(12):
            d = lu.solve(resid(xv, Ab).astype(np.float64))
            xv = xv + d
            last = np.linalg.norm(d) / np.linalg.norm(xv)
            if last < 1e-15:
                break
        return xv, last

    x, last = refine(x, Ab)
    rng = np.random.default_rng(2024)
    k_noise = 0.0
    for _ in range(2):
        Ap = A * (1.0 + EPS * rng.uniform(-1.0, 1.0, A.size))
        xp, _ = refine(x.copy(), Ap.reshape(-1, 6, 6).astype(np.longdouble))
        k_noise = max(k_noise, np.linalg.norm(xp - x) / np.linalg.norm(x))
    bn = np.linalg.norm(b)
    return {"x": x, "rel_res": float(np.linalg.norm(resid(x)) / bn),
            "floor": EPS * np.linalg.norm(abs(S) @ np.abs(x)) / bn,
            "fp64_noise": max(dx[-3:]), "last_dx": last, "k_noise": k_noise,
            "xnorm": np.linalg.norm(x)}


def main(names):
    from gpu_fem_b200 import mesh as M
    cases = {
        "config2_100x50": (lambda: M.plate_config2(100, 50), 1, "plate_config2(100, 50)"),
        "config2_400x200": (lambda: M.plate_config2(), 97, "plate_config2(400, 200)"),
        "box_72x18x6": (lambda: M.box(72, 18, 6), 1, "box(72, 18, 6)"),
    }
    for name in names or cases:
        make, stride, call = cases[name]
        t0 = time.time()
        r = solve(make())
        idx = np.arange(0, r["x"].size, stride, dtype=np.int64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), x=r["x"][idx], idx=idx,
                            xnorm=r["xnorm"], rel_res=r["rel_res"], floor=r["floor"],
                            fp64_noise=r["fp64_noise"], last_dx=r["last_dx"],
                            k_noise=r["k_noise"], mesh=call)
        print(f"{name}: {r['x'].size} DOF, rel_res {r['rel_res']:.2e}, floor {r['floor']:.2e}, "
              f"fp64_noise {r['fp64_noise']:.2e}, k_noise {r['k_noise']:.2e}, "
              f"last correction {r['last_dx']:.1e} "
              f"({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
