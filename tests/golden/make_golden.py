"""Regenerates tests/golden/one_element.json from the CPU oracle.

Inputs are the reference's one-element fixture: xpts of
tests/shell_res/local_utils.h:25-31, vars of tests/shell_res/res.cu:33-36,
perturbations p, p2 of tests/shell_jac/jac.cu:35-39; outputs are the values
the reference's programs print (res TD = p.R, jac TD = p^T K p2, energy, the
residual, the first two rows of K). The oracle's values are pinned by the
complex-step identities in tests/test_oracle_pins.py.
Run: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as po  # noqa: E402

X = np.array([1.0345452 + 2.23123432 * i + 0.323 * i * i for i in range(12)])
u = np.array([(1.4543 + 6.4323 * i) * 1e-6 for i in range(24)])
p = np.array([(-1.4543 + 2.312 * 6.4323 * i) for i in range(24)])
p2 = np.array([(-1.4543 * 1.024343 + 2.812 * -9.4323 * i) for i in range(24)])
d = po.make_data(70e9, 0.3, 0.005)
R = po.element_residual(X, u, d)
_, K = po.element_jacobian(X, u, d)
out = {"xpts": X.tolist(), "vars": u.tolist(), "p": p.tolist(), "p2": p2.tolist(),
       "E": 70e9, "nu": 0.3, "thick": 0.005,
       "res": R.tolist(), "kmat_rows_0_1": K[:2].tolist(),
       "res_TD": float(p @ R), "jac_TD": float(p @ K @ p2),
       "energy": po.element_energy(X, u, d)}
with open(os.path.join(HERE, "one_element.json"), "w") as f:
    json.dump(out, f, indent=1)
print("wrote one_element.json")
