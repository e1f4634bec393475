"""Continuous-batching server: a short Poisson stream of plate and box
requests over the smallest size classes is served to 1e-8; with the coloured
(bitwise-reproducible) assembly scatter a request's displacement is bitwise
the same served in the mix as solved alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_server_stream_and_alone_equals_mix():
    from gpu_fem_b200 import serve
    reqs = serve.poisson_requests(rate=30.0, duration=1.0, seed=99, max_class=2)
    assert len(reqs) >= 10
    srv = serve.Server(budget_gb=8.0, streams=2, max_batch=8, scatter="coloured")
    srv.warm({(r.family, r.cls) for r in reqs})
    srv.keep_results = True
    out = srv.run(reqs)
    assert out["solved"] == len(reqs), (srv.errors, srv.fills, [(r.rid, r.status, r.rel) for r in reqs])
    assert all(r.rel <= 1e-8 for r in reqs)
    assert out["p99_ms"] >= out["p50_ms"] > 0
    r0 = reqs[len(reqs) // 2]
    x_alone = srv.solve_alone(r0)
    x_mix = srv.results[r0.rid]
    assert np.array_equal(x_alone.view(np.uint64), x_mix.view(np.uint64))
