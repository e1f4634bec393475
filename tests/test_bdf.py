"""BDF mesh input (gf_bdf_read, the data TACSMeshLoader hands to
createFromBDF, include/mesh/TACSMeshLoader.h:188-225): a generated mesh
written as NASTRAN bulk data in small-field, large-field and free-field
format, with shuffled, gapped file ids, reads back as the same mesh (nodes
and elements renumbered by ascending file id, tensor node order, natural
BC DOFs). Host only, no GPU."""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M


def _renumbered(m, node_ids, elem_ids):
    """The mesh as the reader numbers it: nodes and elements by file id."""
    norder = np.argsort(node_ids, kind="stable")
    new_of_old = np.empty_like(norder)
    new_of_old[norder] = np.arange(len(norder))
    eorder = np.argsort(elem_ids, kind="stable")
    conn = new_of_old[m.conn[eorder]]
    xpts = m.xpts[norder]
    bcs = np.sort(6 * new_of_old[np.asarray(m.bcs) // 6] + np.asarray(m.bcs) % 6)
    return conn, xpts, bcs


@pytest.mark.parametrize("fmt", ["small", "large", "free"])
def test_bdf_round_trip(tmp_path, fmt):
    from gpu_fem_b200.assembler import read_bdf
    m = M.plate_config2(12, 6)
    rng = np.random.default_rng(3)
    node_ids = rng.permutation(m.num_nodes) * 3 + 7        # shuffled, with gaps
    elem_ids = rng.permutation(m.num_elements) * 2 + 100
    path = str(tmp_path / f"plate_{fmt}.bdf")
    M.write_bdf(m, path, fmt=fmt, node_ids=node_ids, elem_ids=elem_ids, pid=4)
    r = read_bdf(path)
    conn, xpts, bcs = _renumbered(m, node_ids, elem_ids)
    np.testing.assert_array_equal(r["conn"], conn)
    np.testing.assert_array_equal(r["bcs"], bcs)
    # small fields hold 8 characters (about 6 digits), large ones 16 (9 digits
    # as written); free fields carry every digit
    tol = {"small": 1e-5, "large": 1e-8, "free": 0.0}[fmt]
    assert np.abs(r["xpts"] - xpts).max() <= tol * max(1.0, np.abs(xpts).max())
    assert (r["component"] == 4).all()


def test_bdf_nastran_reals_and_continuations(tmp_path):
    from gpu_fem_b200.assembler import read_bdf
    text = "\n".join([
        "$ two elements",
        "BEGIN BULK",
        "GRID           1       0      0.      0.      0.",
        "GRID           2       0     1.0      0.  1.5-3",
        "GRID,3,0,0.0,1.0,-2.+0",
        "GRID*                  4               0              1.              1.",
        "*                     0.",
        "GRID           5       0      2.      0.      0.",
        "GRID           6       0      2.      1.      0.",
        "CQUAD4        11       1       1       2       4       3",
        "CQUAD4        10       2       2       5       6       4",
        "SPC            1       1  123456      0.       3     345      0.",
        "ENDDATA",
    ])
    path = tmp_path / "two.bdf"
    path.write_text(text)
    r = read_bdf(str(path))
    assert r["xpts"][1, 2] == pytest.approx(1.5e-3)
    assert r["xpts"][2, 2] == pytest.approx(-2.0)
    np.testing.assert_array_equal(r["xpts"][3], [1.0, 1.0, 0.0])
    # elements sorted by id (10 before 11); G1 G2 G3 G4 -> G1 G2 G4 G3
    np.testing.assert_array_equal(r["conn"], [[1, 4, 3, 5], [0, 1, 2, 3]])
    np.testing.assert_array_equal(r["component"], [2, 1])
    np.testing.assert_array_equal(r["bcs"], list(range(6)) + [6 * 2 + 2, 6 * 2 + 3, 6 * 2 + 4])


def test_bdf_rejects_non_shell_elements(tmp_path):
    from gpu_fem_b200 import _lib as L
    from gpu_fem_b200.assembler import read_bdf
    path = tmp_path / "tri.bdf"
    path.write_text("BEGIN BULK\nGRID,1,0,0.,0.,0.\nGRID,2,0,1.,0.,0.\nGRID,3,0,0.,1.,0.\n"
                    "CTRIA3,1,1,1,2,3\nENDDATA\n")
    with pytest.raises(L.GpuFemError) as e:
        read_bdf(str(path))
    assert e.value.status == L.GF_INVALID_ARG
    assert "CTRIA3" in str(e.value)
