"""Node orderings on the host (gf_order_nodes): RCM bit-exact against the
oracle's restatement of TacsComputeRCMOrder (include/linalg/reordering_utils.h
:189-291), and the deterministic q-ordering (examples/iterative/gmres.cu
:159-215 with a fixed seed instead of std::random_device) bit-exact against
the oracle's own restatement; q-ordering only permutes positions within its
windows of floor(bandwidth / p) consecutive RCM positions."""
import numpy as np
import pytest

from gpu_fem_b200 import mesh as M


@pytest.mark.parametrize("p, seed", [(1.0, 0), (0.5, 7), (2.0, 123456789)])
def test_qorder_matches_oracle_and_stays_in_windows(oracle, p, seed):
    from gpu_fem_b200.assembler import order_nodes
    m = M.plate_config2(30, 14)
    rowp, cols = oracle.bsr_pattern(m.conn, m.num_nodes)
    rcm = oracle.rcm(rowp, cols, 0, 1)
    np.testing.assert_array_equal(order_nodes(m.conn, m.num_nodes, "rcm"), rcm)
    q = order_nodes(m.conn, m.num_nodes, "qorder", qorder_p=p, qorder_seed=seed)
    np.testing.assert_array_equal(q, oracle.qorder(rowp, cols, rcm, p, seed))
    assert np.array_equal(np.sort(q), np.arange(m.num_nodes))   # a permutation
    r2, c2 = oracle.permute_pattern(rowp, cols, rcm)
    rows = np.repeat(np.arange(m.num_nodes), np.diff(r2))
    width = max(1, int(np.abs(rows - c2).max() / p))
    assert (q // width == rcm // width).all()                  # same window
    assert (q != rcm).sum() > m.num_nodes // 2                  # actually shuffled
    # deterministic, and the seed matters
    np.testing.assert_array_equal(q, order_nodes(m.conn, m.num_nodes, "qorder", qorder_p=p,
                                                 qorder_seed=seed))
    assert not np.array_equal(q, order_nodes(m.conn, m.num_nodes, "qorder", qorder_p=p,
                                             qorder_seed=seed + 1))
