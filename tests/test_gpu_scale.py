"""Displacements of the scale meshes against FP64 direct-solve goldens.

Goldens (tests/golden/*.npz, written offline by tests/golden/make_scale_golden.py
with SuperLU in symmetric mode plus iterative refinement with extended-
precision residuals, settled to about 1e-11) stand in for
the reference's direct solve (examples/plate_demo/linear_static.cu:12-73).
Each mesh is assembled, factored (ILU(k) in the stated ordering) and solved
with right-preconditioned GMRES on the GPU, once with FP64 factors and once
with FP32 factors inside FP64 GMRES (the mixed mode), and the displacement
error against the golden is checked and printed per solve.

Gate: ||x - x_golden|| / ||x_golden|| <= max(1e-8, 3 * max(fp64_noise, k_noise)).
Both noise figures are computed with each golden: fp64_noise is how far an
exactly factored FP64 solve still moves under refinement with FP64
residuals, and k_noise is how far x moves when every entry of K is perturbed
by one rounding (a relative eps), i.e. how precisely any FP64 assembly of K
defines x. For the plates of the batch workload and for the box both are far
below 1e-8 (box: 4.7e-12 and 8.2e-12) and the gate is 1e-8. The jittered
cantilever (2 x 1 m, t = 4 mm, one edge clamped) is the exception: one
rounding of K moves its x by 1.0e-8 at 100 x 50 and by 8.2e-8 at its stated
400 x 200, so two correct FP64 assemblies and solves can differ by that much
and the gate there is 3.1e-8 and 2.5e-7. Its relative residual cannot go
below eps || |K| |x| || / ||b|| (3.0e-7 and 4.8e-6: the residual of x rounded
to FP64) for any solver, so its GMRES tolerance is that floor; the
workload's 1e-8 residual is out of reach for it in FP64. At 400 x 200 block
ILU(k)-GMRES does not converge at all (ILU(8), RCM or natural ordering,
stalls near 0.99 on the GPU and in the CPU oracle alike), so that size has a
golden (config2_400x200.npz) but no solve here.
"""
import os

import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: g[k] for k in g.files}


def _solve(mesh, ordering, fill, precision, rtol, restart=100, max_iters=20000):
    import torch
    from gpu_fem_b200.assembler import (ElementAssembler, ILUk_Preconditioner, SolveOptions,
                                        createBsrMat, gmres_solve)
    A = ElementAssembler.from_mesh(mesh, ordering=ordering)
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    P = ILUk_Preconditioner(A, fill_level=fill, precision=precision)
    P.factor(K)
    b = torch.tensor(mesh.loads, device="cuda")
    x = torch.zeros_like(b)
    st, stats = gmres_solve(A, K, P, b, x, SolveOptions(restart=restart, max_iters=max_iters,
                                                        rtol=rtol, side=1))
    return x.cpu().numpy(), stats


def _check(name, x, g, stats, label):
    idx = g["idx"]
    err = np.linalg.norm(x[idx] - g["x"]) / np.linalg.norm(g["x"])
    bound = max(1e-8, 3.0 * max(float(g["fp64_noise"]), float(g["k_noise"])))
    print(f"{name} {label}: rel residual {stats['rel_residual']:.2e}, "
          f"{stats['iterations']} GMRES steps, displacement error {err:.2e} (gate {bound:.2e})")
    assert err <= bound, (name, label, err, bound, stats)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cantilever_100x50_matches_direct_solve(precision):
    g = _golden("config2_100x50")
    x, stats = _solve(M.plate_config2(100, 50), "rcm", 8, precision, rtol=float(g["floor"]))
    _check("cantilever 100x50", x, g, stats, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_box_72x18x6_matches_direct_solve(precision):
    g = _golden("box_72x18x6")
    x, stats = _solve(M.box(72, 18, 6), "rcm", 12, precision, rtol=1e-9)
    _check("box 72x18x6", x, g, stats, precision)

