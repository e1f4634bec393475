"""The drop-in boundary, run: the C++ facade driver (tests/drivers/linear_static.cpp,
the reference's linear_static.cu call sequence: template composition,
ElementAssembler, createBsrMat, add_jacobian, apply_bcs,
CUSPARSE::direct_LU_solve_old, ILUk_Preconditioner + GMRES, add_energy) and
the C driver (tests/drivers/c_abi_solve.c, the bare C ABI) are built, run as
separate programs on config 1 (10 x 10 clamped plate, t = 5 mm, 1 kPa), and
their outputs are compared with the CPU oracle:
- the assembled K with the Dirichlet rows / columns: entries within 1e-12
  of max |K| of the oracle's, pattern and permutation bit-exact;
- the direct block LU solve and the ILU(2)-GMRES solve (to 1e-10): within
  1e-10 and 1e-8 of a dense FP64 solve;
- the strain energy at the solution equals 1/2 b^T x within 1e-10.
"""
import os
import subprocess

import numpy as np
import pytest

from gpu_fem_b200 import mesh as M
from test_boundary_compile import build_driver

pytestmark = pytest.mark.gpu


def _write_mesh(path, m):
    with open(path, "wb") as f:
        np.array([m.num_nodes, m.num_elements, len(m.bcs)], np.int32).tofile(f)
        np.array([m.E, m.nu], np.float64).tofile(f)
        np.ascontiguousarray(m.conn, np.int32).tofile(f)
        np.ascontiguousarray(m.xpts, np.float64).tofile(f)
        np.ascontiguousarray(m.bcs, np.int32).tofile(f)
        np.broadcast_to(np.asarray(m.thick, np.float64), (m.num_elements,)).tofile(f)
        np.ascontiguousarray(m.loads, np.float64).tofile(f)


def _read(prefix, m):
    pat = np.fromfile(prefix + ".pattern", np.int32)
    nn, nnzb = pat[0], pat[1]
    rowp = pat[2:3 + nn]
    cols = pat[3 + nn:3 + nn + nnzb]
    perm = pat[3 + nn + nnzb:3 + 2 * nn + nnzb]
    return (rowp, cols, perm, np.fromfile(prefix + ".K", np.float64),
            np.fromfile(prefix + ".x_direct", np.float64),
            np.fromfile(prefix + ".x_gmres", np.float64), np.fromfile(prefix + ".info", np.float64))


@pytest.mark.parametrize("driver", ["linear_static.cpp", "c_abi_solve.c"])
def test_driver_runs_and_matches_oracle(oracle, driver, tmp_path):
    exe = build_driver(driver, tmp_path)
    m = M.plate_config1()
    mesh_path = str(tmp_path / "mesh.bin")
    _write_mesh(mesh_path, m)
    prefix = str(tmp_path / "out")
    env = dict(os.environ)
    args = [exe, mesh_path, prefix]
    if driver.endswith(".cpp"):  # also TACSMeshLoader + createFromBDF
        M.write_bdf(m, str(tmp_path / "mesh.bdf"), fmt="free")
        args.append(str(tmp_path / "mesh.bdf"))
    r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    rowp, cols, perm, K, x_direct, x_gmres, info = _read(prefix, m)
    # the oracle in the same ordering
    rowp_o, cols_o, vals_o, _, _ = oracle.assemble_jacobian(m, perm=perm)
    oracle.apply_bcs_mat(rowp_o, cols_o, vals_o, perm, m.bcs)
    np.testing.assert_array_equal(rowp, rowp_o)
    np.testing.assert_array_equal(cols, cols_o)
    rowp0, cols0 = oracle.bsr_pattern(m.conn, m.num_nodes)
    np.testing.assert_array_equal(perm, oracle.rcm(rowp0, cols0, 0, 1))
    assert np.abs(K - vals_o).max() <= 1e-12 * np.abs(vals_o).max()
    b = np.zeros(m.num_dof)
    b.reshape(-1, 6)[perm] = m.loads.reshape(-1, 6)
    xd = oracle.dense_solve(oracle.bsr_to_dense(rowp_o, cols_o, vals_o), b)
    xd = xd.reshape(-1, 6)[perm].ravel()
    e_direct = np.linalg.norm(x_direct - xd) / np.linalg.norm(xd)
    e_gmres = np.linalg.norm(x_gmres - xd) / np.linalg.norm(xd)
    print(f"{driver}: direct error {e_direct:.2e}, GMRES error {e_gmres:.2e}, info {info}")
    assert e_direct <= 1e-10, e_direct
    assert e_gmres <= 1e-8, e_gmres
    if driver.endswith(".cpp"):
        U = info[0]
        half_bx = 0.5 * float(m.loads @ x_direct)
        assert abs(U - half_bx) <= 1e-10 * abs(half_bx), (U, half_bx)
