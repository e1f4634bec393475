"""Symbolic setup on the GPU. ILU(k) symbolic factorization (gf_precond_create ->
iluk_pattern_gpu): the pattern is bit-exact against the oracle's restatement
of computeILUk (include/linalg/bsr_utils.h:678-807) for natural, RCM and
q-ordered plates, a stiffened box and the complete factor (GF_FILL_FULL),
and gf_precond_setup_info reports that the GPU computed it. Node pattern and
elemIndMap of gf_assembler_create, bit-exact, with gf_assembler_setup_info."""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _plate(nx, ny, t=0.003):
    return M.plate(nx, ny, 1.0, ny / nx, lambda x, y: t + 0 * x, "all_edges",
                   lambda q: 1e3 + 0 * q[:, 0], name=f"plate_{nx}x{ny}")


@pytest.mark.parametrize("case,fills", [
    (("plate", 64, 32, "natural"), [1, 2, 4, 8, 16]),
    (("plate", 48, 40, "rcm"), [1, 3, 6, 12]),
    (("plate", 40, 24, "qorder"), [2, 5]),
    (("box", None, None, "rcm"), [2, 8]),
])
def test_gpu_iluk_pattern_matches_oracle(case, fills):
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner
    from oracle import pyoracle as po
    kind, nx, ny, ordering = case
    mesh = _plate(nx, ny) if kind == "plate" else M.box(18, 6, 4)
    kw = {"qorder_p": 2.0, "qorder_seed": 7} if ordering == "qorder" else {}
    A = ElementAssembler.from_mesh(mesh, ordering=ordering, **kw)
    bd = A.getBsrData()
    for fill in fills:
        P = ILUk_Preconditioner(A, fill_level=fill, precision="fp64")
        info = P.setup_info()
        assert info["symbolic_on_gpu"], (case, fill, info)
        r, c, _ = P.get()
        ro, co = po.iluk_pattern(bd["rowPtr"], bd["colPtr"], fill)
        np.testing.assert_array_equal(r, ro)
        np.testing.assert_array_equal(c, co)


def test_gpu_complete_factor_pattern():
    """GF_FILL_FULL: every fill entry kept, the pattern of the complete block
    LU (the oracle's full-fill count)."""
    from gpu_fem_b200 import _lib as L
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner
    from oracle import pyoracle as po
    A = ElementAssembler.from_mesh(_plate(24, 12), ordering="rcm")
    bd = A.getBsrData()
    P = ILUk_Preconditioner(A, fill_level=L.GF_FILL_FULL, precision="fp64")
    assert P.setup_info()["symbolic_on_gpu"]
    r, c, _ = P.get()
    assert r[-1] == po.full_fill_count(bd["rowPtr"], bd["colPtr"])


@pytest.mark.parametrize("kind,ordering", [("plate", "natural"), ("plate", "rcm"),
                                           ("jittered", "rcm"), ("box", "rcm")])
def test_gpu_node_pattern_and_elem_map_match_oracle(kind, ordering):
    """Node pattern (get_row_col_ptrs) and elemIndMap (get_elem_ind_map) built
    on the GPU by gf_assembler_create: bit-exact against the oracle in the
    solver ordering."""
    from gpu_fem_b200.assembler import ElementAssembler
    from oracle import pyoracle as po
    mesh = {"plate": lambda: _plate(40, 24), "jittered": lambda: M.plate_config2(30, 15),
            "box": lambda: M.box(18, 6, 4)}[kind]()
    A = ElementAssembler.from_mesh(mesh, ordering=ordering)
    info = A.setup_info()
    assert info["pattern_on_gpu"] and info["elem_map_on_gpu"], info
    bd = A.getBsrData()
    r0, c0 = po.bsr_pattern(mesh.conn, mesh.num_nodes)
    rp, cp = po.permute_pattern(r0, c0, bd["perm"])[:2]
    np.testing.assert_array_equal(bd["rowPtr"], rp)
    np.testing.assert_array_equal(bd["colPtr"], cp)
    np.testing.assert_array_equal(bd["elemIndMap"], po.elem_ind_map(mesh.conn, rp, cp, bd["perm"]))
