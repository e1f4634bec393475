"""gf_precond_apply_noalloc against gf_precond_apply.

The no-allocation variant keeps the intermediate vector of the two
triangular sweeps in a fixed device array instead of the preconditioner's
own buffers. Both entry points are called through the C ABI on the same
factors, twice in a row with different right-hand sides (the second call
finds the first call's contents in the shared array), and must agree to the
tolerance the preconditioner-apply test uses. Sizes above the array's
capacity are refused before anything runs.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _factored(mesh, fill, precision, ordering="rcm", sweep="auto"):
    import torch
    from gpu_fem_b200.assembler import ElementAssembler, ILUk_Preconditioner, createBsrMat
    A = ElementAssembler.from_mesh(mesh, ordering=ordering)
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    P = ILUk_Preconditioner(A, fill_level=fill, precision=precision, sweep=sweep)
    P.factor(K)
    torch.cuda.synchronize()
    return A, K, P


def _case(name):
    """single_cta: 24x12 jittered cantilever, RCM, ILU(2), level-synchronous
    sweeps on one CTA. split: 256x128 clamped plate, natural ordering,
    ILU(6), 33,153 nodes (below the array's 43,690-node capacity), 26 rows a
    level: with FP32 factors the level-synchronous sweeps split every chunk
    over a 2-CTA cluster, so the intermediate vector in the fixed array is
    written by two CTAs; with FP64 factors every level spans two chunks of
    one CTA. dataflow: the same plate with the dataflow sweeps."""
    plate = M.plate(256, 128, 1.0, 0.5, lambda x, y: 0.002 + 0 * x, "all_edges",
                    lambda q: 1e3 + 0 * q[:, 0])
    return {"single_cta": (M.plate_config2(24, 12), 2, "rcm", "level", 1),
            "split": (plate, 6, "natural", "level", 2),
            "dataflow": (plate, 6, "natural", "dataflow", 1)}[name]


@pytest.mark.parametrize("case", ["single_cta", "split", "dataflow"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_apply_matches_apply_twice(precision, case):
    import torch
    from gpu_fem_b200 import _lib as L
    lib = L.lib()
    mesh, fill, ordering, sweep, nsplit = _case(case)
    A, K, P = _factored(mesh, fill, precision, ordering, sweep)
    assert P.sweeps()["L"] == sweep
    ns = [C.c_int32(), C.c_int32()]
    assert lib.gf_precond_layout(P.h, C.byref(ns[0]), C.byref(ns[1]), None, None, None) == L.GF_OK
    if case == "split" and precision == "fp64":
        nsplit = 1  # two one-CTA chunks a level (see _case)
    assert (ns[0].value, ns[1].value) == (nsplit, nsplit)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(7)
    for call in range(2):
        r = torch.tensor(rng.standard_normal(mesh.num_dof), device="cuda")
        z_ref = torch.zeros_like(r)
        z_new = torch.full_like(r, float("nan"))
        st = lib.gf_precond_apply(P.h, C.c_void_p(r.data_ptr()), C.c_void_p(z_ref.data_ptr()),
                                  stream)
        assert st == L.GF_OK, L.lib().gf_last_error()
        st = lib.gf_precond_apply_noalloc(P.h, C.c_void_p(r.data_ptr()),
                                          C.c_void_p(z_new.data_ptr()), stream)
        assert st == L.GF_OK, L.lib().gf_last_error()
        assert lib.gf_precond_status(P.h, stream) == L.GF_OK  # no bounded wait ran out
        a, b = z_ref.cpu().numpy(), z_new.cpu().numpy()
        assert np.isfinite(b).all(), call
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max(), (call, np.abs(a - b).max())


def test_noalloc_apply_refuses_problems_above_capacity():
    import torch
    from gpu_fem_b200 import _lib as L
    lib = L.lib()
    # 211 x 211 nodes: 6 * 44521 = 267126 doubles > 262144
    mesh = M.plate(210, 210, 1.0, 1.0, lambda x, y: 0.005 + 0 * x, "all_edges",
                   lambda q: 1e3 + 0 * q[:, 0])
    assert 6 * mesh.num_nodes > 262144
    A, K, P = _factored(mesh, 0, "fp64")
    r = torch.ones(mesh.num_dof, dtype=torch.float64, device="cuda")
    z = torch.zeros_like(r)
    st = lib.gf_precond_apply_noalloc(P.h, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == L.GF_INVALID_ARG
    msg = lib.gf_last_error()
    msg = msg.decode() if isinstance(msg, bytes) else msg
    assert "262144" in msg and str(6 * mesh.num_nodes) in msg
    torch.cuda.synchronize()
    assert float(z.abs().max()) == 0.0  # nothing ran
