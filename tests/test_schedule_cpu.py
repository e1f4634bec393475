"""Host logic: the scatter schedule restated by the oracle is a valid
colouring with unique first touches; RCM, pattern and ILU(k) patterns of the
oracle agree with independent restatements."""
import numpy as np
import scipy.sparse as sp

from gpu_fem_b200 import mesh as M
from oracle.schedule import schedule


def _check_schedule(mesh, oracle, chunk=8):
    rowp, cols = oracle.bsr_pattern(mesh.conn, mesh.num_nodes)
    perm = np.arange(mesh.num_nodes, dtype=np.int32)
    emap = oracle.elem_ind_map(mesh.conn, rowp, cols, perm)
    s = schedule(mesh.conn, mesh.num_nodes, emap, chunk_size=chunk)
    conn = mesh.conn
    # chunk sizes
    counts = np.bincount(s["elem_chunk"])
    assert counts.max() <= chunk
    # same-coloured chunks never share a node; same-coloured elements of a chunk neither
    owner = {}
    for e in range(conn.shape[0]):
        for n in conn[e]:
            owner.setdefault(int(n), []).append(e)
    for n, es in owner.items():
        cc = {}
        for e in es:
            c = s["elem_chunk"][e]
            col = s["chunk_color"][c]
            cc.setdefault(col, set()).add(c)
            assert len(cc[col]) == 1
        pairs = {}
        for e in es:
            key = (s["elem_chunk"][e], s["elem_color"][e])
            assert key not in pairs
            pairs[key] = e
    # every block has exactly one first touch
    ft = s["first_touch"]
    first = np.zeros(len(cols), np.int32)
    for e in range(conn.shape[0]):
        for k in range(16):
            if (ft[e] >> k) & 1:
                first[emap[16 * e + k]] += 1
    assert (first == 1).all()
    return s


def test_schedule_plate(oracle):
    s = _check_schedule(M.plate_config2(40, 20), oracle)
    assert s["num_chunk_colors"] <= 8


def test_schedule_box(oracle):
    _check_schedule(M.box(nx=18, ny=6, nz=4, nribs=4), oracle)


def test_pattern_matches_scipy(oracle):
    mesh = M.plate_config2(12, 7)
    rowp, cols = oracle.bsr_pattern(mesh.conn, mesh.num_nodes)
    n = mesh.num_nodes
    r, c = [], []
    for e in mesh.conn:
        for a in e:
            for b in e:
                r.append(a)
                c.append(b)
    A = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    np.testing.assert_array_equal(rowp, A.indptr)
    np.testing.assert_array_equal(cols, A.indices)


def test_rcm_is_reversed_bfs(oracle):
    mesh = M.plate_config2(10, 6)
    rowp, cols = oracle.bsr_pattern(mesh.conn, mesh.num_nodes)
    rcm = oracle.rcm(rowp, cols, 0, 1)
    n = mesh.num_nodes
    # independent BFS restatement (neighbours in column order, no degree sort)
    order, seen = [0], {0}
    head = 0
    while head < len(order):
        v = order[head]
        head += 1
        for w in cols[rowp[v]:rowp[v + 1]]:
            if int(w) not in seen:
                seen.add(int(w))
                order.append(int(w))
    expect = np.empty(n, np.int32)
    for i, v in enumerate(order):
        expect[v] = n - 1 - i
    np.testing.assert_array_equal(rcm, expect)


def test_iluk_pattern_levels(oracle):
    mesh = M.plate_config2(10, 6)
    rowp, cols = oracle.bsr_pattern(mesh.conn, mesh.num_nodes)
    r0, c0 = oracle.iluk_pattern(rowp, cols, 0)
    np.testing.assert_array_equal(r0, rowp)
    np.testing.assert_array_equal(c0, cols)
    prev = len(cols)
    for k in (1, 2, 3):
        rk, ck = oracle.iluk_pattern(rowp, cols, k)
        assert len(ck) > prev
        prev = len(ck)
    # full fill equals ILU(n)
    rk, ck = oracle.iluk_pattern(rowp, cols, 10 ** 6)
    assert len(ck) == oracle.full_fill_count(rowp, cols)
