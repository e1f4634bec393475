"""createFromBDF on the GPU: an assembler built from a free-field BDF file of
a mesh (exact coordinates) assembles bitwise the same Jacobian and solves to
bitwise the same displacements as the assembler built from the mesh arrays
(include/assembler.h:92-115)."""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu


def test_create_from_bdf_matches_direct_assembler(tmp_path):
    import torch
    from gpu_fem_b200.assembler import (ElementAssembler, ILUk_Preconditioner, SolveOptions,
                                        createBsrMat, gmres_solve)
    m = M.plate_config1()
    path = str(tmp_path / "plate.bdf")
    M.write_bdf(m, path, fmt="free")
    out = []
    for A in (ElementAssembler.from_mesh(m, ordering="rcm"),
              ElementAssembler.createFromBDF(path, E=m.E, nu=m.nu, thick=float(m.thick[0]),
                                             ordering="rcm")):
        K = createBsrMat(A)
        A.add_jacobian(None, K, fuse_bcs=True)
        P = ILUk_Preconditioner(A, fill_level=2)
        P.factor(K)
        b = torch.tensor(m.loads, device="cuda")
        x = torch.zeros_like(b)
        st, stats = gmres_solve(A, K, P, b, x, SolveOptions(rtol=1e-10, restart=200))
        assert stats["rel_residual"] <= 1e-10
        out.append((K.values_host(), x.cpu().numpy()))
    assert np.array_equal(out[0][0].view(np.uint64), out[1][0].view(np.uint64))
    assert np.array_equal(out[0][1].view(np.uint64), out[1][1].view(np.uint64))
