"""Bounded device-side waits report GF_TIMEOUT and leave the context usable.

The dataflow factorization waits, bounded, for the completion flag of every
row a step reads; the split (level-synchronous) sweeps meet the partner CTA
of their cluster once per chunk on mbarriers with bounded waits; the
dataflow sweep waits, bounded, for the result tags of the rows each row
multiplies. The tests shorten the bound to 200 us and switch on
gf_test_set_waits' failure injection: the factorization never publishes the
first row of its order, CTA rank 1 of a sweep cluster skips its meeting
arrivals, and the dataflow sweep's warp 0 never publishes its rows, so the
waits run out. The launches record a timeout (the first wait that runs out
ends the factorization's other waits), both CTAs of a cluster still meet on
the final cluster barrier, every CTA lets its copies in flight land,
and the host reads GF_TIMEOUT from gf_precond_factor, gf_precond_status after
an apply, and gf_gmres_solve. With the default bound restored, the same
objects factor and solve correctly. No wait is removed, so nothing can hang,
and nothing faults.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_fem_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _status(P):
    import torch
    from gpu_fem_b200 import _lib as L
    return L.lib().gf_precond_status(P.h, C.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("sweep", ["level", "dataflow"])
def test_timeout_reported_and_context_usable(sweep):
    import torch
    from gpu_fem_b200 import _lib as L
    from gpu_fem_b200.assembler import (ElementAssembler, ILUk_Preconditioner, SolveOptions,
                                        createBsrMat, gmres_solve)
    lib = L.lib()
    mesh = M.plate(160, 80, 1.0, 0.5, lambda x, y: 0.002 + 0 * x, "all_edges",
                   lambda q: 1e3 + 0 * q[:, 0])
    A = ElementAssembler.from_mesh(mesh, ordering="natural")
    K = createBsrMat(A)
    A.add_jacobian(None, K, fuse_bcs=True)
    P = ILUk_Preconditioner(A, fill_level=6, precision="fp64", sweep=sweep)
    lay = P.layout()
    assert lay["fac_ctas"] == 128  # the dataflow factorization's CTAs
    assert P.sweeps()["L"] == sweep
    if sweep == "level":  # both sweeps split every chunk over two CTAs
        assert (lay["nsplit_L"], lay["nsplit_U"]) == (2, 2)
    P.factor(K)
    r = torch.tensor(np.random.default_rng(3).standard_normal(mesh.num_dof), device="cuda")
    z_ok = torch.zeros_like(r)
    P.apply(r, z_ok)
    assert _status(P) == L.GF_OK
    b = torch.tensor(mesh.loads, device="cuda")
    opts = SolveOptions(restart=100, max_iters=3000, rtol=1e-8, side=1)
    torch.cuda.synchronize()
    try:
        L.check(lib.gf_test_set_waits(200_000, 1), "set_waits")
        # dataflow factorization: the rows that read the unpublished row time out
        with pytest.raises(L.GpuFemError) as err:
            P.factor(K)
        assert err.value.status == L.GF_TIMEOUT
        # split sweeps: the chunk meetings run out; the apply itself does
        # not wait for the GPU, the status query reports it
        z = torch.zeros_like(r)
        P.apply(r, z)
        assert _status(P) == L.GF_TIMEOUT
        assert _status(P) == L.GF_OK  # read and cleared
        x = torch.zeros_like(b)
        st, stats = gmres_solve(A, K, P, b, x, opts, raise_on_fail=False)
        assert st == L.GF_TIMEOUT and stats["status"] == L.GF_TIMEOUT
    finally:
        L.check(lib.gf_test_set_waits(0, 0), "restore waits")
    torch.cuda.synchronize()
    # the context and the objects are still usable
    P.factor(K)
    z = torch.zeros_like(r)
    P.apply(r, z)
    assert _status(P) == L.GF_OK
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy().view(np.uint64), z_ok.cpu().numpy().view(np.uint64))
    x = torch.zeros_like(b)
    st, stats = gmres_solve(A, K, P, b, x, opts)
    assert st == L.GF_OK and stats["rel_residual"] <= 1e-8, stats
