"""Pins of the CPU oracle against the reference's own checks.

The reference has no stored expected values; its tests print numbers from
(1) complex-step identities (tests/shell_res/res_cs.cu, tests/shell_jac/jac-cs.cu),
(2) a 2-element fill-in known answer (examples/basic_shell/test_fill_in.cu:24-29),
(3) the Navier simply-supported plate (examples/plate_demo/_plate_utils.h:18-38).
Each is asserted here, plus the committed golden vectors of the one-element
fixture (tests/golden/one_element.json, made by tests/golden/make_golden.py).
"""
import json
import os

import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def fixture():
    X = np.array([1.0345452 + 2.23123432 * i + 0.323 * i * i for i in range(12)])
    u = np.array([(1.4543 + 6.4323 * i) * 1e-6 for i in range(24)])
    p = np.array([(-1.4543 + 2.312 * 6.4323 * i) for i in range(24)])
    p2 = np.array([(-1.4543 * 1.024343 + 2.812 * -9.4323 * i) for i in range(24)])
    return X, u, p, p2


def test_mt19937_64_known_answer():
    # C++ standard [rand.predef]: the 10000th output of a default-constructed
    # mt19937_64 is 9981545732273789042.
    assert int(M.MT19937_64(5489).raw(10000)[-1]) == 9981545732273789042


def test_complex_step_residual(oracle):
    X, u, p, _ = fixture()
    d = oracle.make_data(70e9, 0.3, 0.005)
    h = 1e-30
    R = oracle.element_residual(X, u, d)
    U = oracle.element_energy_cs(X, u, p * h, d)
    assert abs(p @ R - U.imag / h) <= 1e-12 * abs(p @ R)


def test_complex_step_jacobian(oracle):
    X, u, p, p2 = fixture()
    d = oracle.make_data(70e9, 0.3, 0.005)
    h = 1e-30
    _, K = oracle.element_jacobian(X, u, d)
    Rc = oracle.element_residual_cs(X, u, p * h, d)
    lhs = p @ K @ p2
    assert abs(lhs - (p2 @ Rc).imag / h) <= 1e-12 * abs(lhs)


def test_linearity_symmetry_energy(oracle):
    X, u, _, _ = fixture()
    d = oracle.make_data(70e9, 0.3, 0.005)
    R = oracle.element_residual(X, u, d)
    R2, K = oracle.element_jacobian(X, u, d)
    assert np.abs(K - K.T).max() <= 1e-14 * np.abs(K).max()
    assert np.abs(K @ u - R).max() <= 1e-13 * np.abs(R).max()
    assert np.abs(R2 - R).max() <= 1e-13 * np.abs(R).max()
    assert abs(oracle.element_energy(X, u, d) - 0.5 * u @ K @ u) <= 1e-12 * abs(u @ K @ u)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_rigid_translation_is_zero_energy(oracle, k):
    X = np.array([0, 0, 0, 1.1, 0.05, 0.02, -0.03, 0.9, 0.0, 1.0, 1.0, 0.1])
    d = oracle.make_data(70e9, 0.3, 0.004)
    _, K = oracle.element_jacobian(X, np.zeros(24), d)
    t = np.zeros(24)
    t[k::6] = 1.0
    assert np.abs(K @ t).max() <= 1e-9 * np.abs(K).max()


def test_fill_in_known_answer(oracle):
    conn = np.array([[0, 1, 2, 3], [1, 3, 4, 5]], np.int32)
    rowp, cols = oracle.bsr_pattern(conn, 6)
    assert len(cols) == 28
    np.testing.assert_array_equal(rowp, [0, 4, 10, 14, 20, 24, 28])
    assert oracle.full_fill_count(rowp, cols) == 32


def test_golden_one_element(oracle):
    with open(os.path.join(GOLDEN, "one_element.json")) as f:
        g = json.load(f)
    X, u, p, p2 = fixture()
    d = oracle.make_data(70e9, 0.3, 0.005)
    R = oracle.element_residual(X, u, d)
    _, K = oracle.element_jacobian(X, u, d)
    np.testing.assert_allclose(R, g["res"], rtol=0, atol=1e-13 * np.abs(g["res"]).max())
    np.testing.assert_allclose(K[:2], np.array(g["kmat_rows_0_1"]), rtol=0,
                               atol=1e-13 * np.abs(K).max())
    assert abs(p @ R - g["res_TD"]) <= 1e-12 * abs(g["res_TD"])
    assert abs(p @ K @ p2 - g["jac_TD"]) <= 1e-12 * abs(g["jac_TD"])
    assert abs(oracle.element_energy(X, u, d) - g["energy"]) <= 1e-12 * g["energy"]


def _navier_mesh(n, a=1.0, t=0.005, Q=1.0e3):
    """Simply supported plate of createPlateAssembler (_plate_utils.h:47-83)
    under q = Q sin(pi x/a) sin(pi y/b) with consistent nodal loads."""
    mesh = M.plate(n, n, a, a, lambda x, y: t + 0 * x, "all_edges",
                   lambda q: Q * np.sin(np.pi * q[:, 0] / a) * np.sin(np.pi * q[:, 1] / a))
    nnx = n + 1
    bcs = list(range(6))
    for ix in range(1, nnx):
        bcs += [6 * ix + 1, 6 * ix + 2]
    for iy in range(1, nnx):
        bcs += [6 * (nnx * iy), 6 * (nnx * iy) + 2, 6 * (nnx * iy + nnx - 1) + 2]
    for ix in range(1, nnx - 1):
        bcs.append(6 * (nnx * (nnx - 1) + ix) + 2)
    mesh.bcs = np.array(sorted(set(bcs)), np.int32)
    mesh.loads[mesh.bcs] = 0.0
    return mesh


def test_navier_plate(oracle):
    n, a, t, Q = 16, 1.0, 0.005, 1.0e3
    mesh = _navier_mesh(n, a, t, Q)
    rowp, cols, vals, _, perm = oracle.assemble_jacobian(mesh)
    oracle.apply_bcs_mat(rowp, cols, vals, perm, mesh.bcs)
    x = oracle.dense_solve(oracle.bsr_to_dense(rowp, cols, vals), mesh.loads)
    D = 70e9 * t ** 3 / (12 * (1 - 0.3 ** 2))
    w_exact = Q / (D * np.pi ** 4 * (4.0 / a ** 4))
    w_center = x[6 * ((n // 2) * (n + 1) + n // 2) + 2]
    assert abs(w_center - w_exact) <= 0.03 * w_exact
