"""Oracle restatement of the coloured scatter schedule (pure Python).

TEST INFRASTRUCTURE. The CUDA assembly orders its 6x6 block scatter by this
project's own deterministic schedule (there is no colouring in the
reference); this file restates that specification independently so tests
can compare chunks, colours and first-touch masks bit-exactly:

 1. Chunks (one warp's work): seeds in ascending element order; a chunk
    grows breadth-first over elements sharing a node (for each dequeued
    element, its nodes in element-local order, each node's elements in
    ascending order) until it holds `chunk_size` elements.
 2. Chunk colours: greedy in chunk order; smallest colour not used by an
    already-coloured chunk sharing a node.
 3. An element's colour is its position in its chunk (the warp processes a
    chunk's elements one after another).
 4. First touch of a block / node: the toucher with the smallest
    (chunk colour, position).
Small meshes only (pure-Python loops).
"""
from __future__ import annotations

import numpy as np


def schedule(conn, nnodes, emap, chunk_size=8, max_ec=15):
    conn = np.asarray(conn).reshape(-1, 4)
    ne = conn.shape[0]
    node_elems = [[] for _ in range(nnodes)]
    for e in range(ne):
        for a in range(4):
            node_elems[conn[e, a]].append(e)
    elem_chunk = [-1] * ne
    chunks = []
    for seed in range(ne):
        if elem_chunk[seed] >= 0:
            continue
        c = len(chunks)
        members = [seed]
        elem_chunk[seed] = c
        head = 0
        while head < len(members) and len(members) < chunk_size:
            e = members[head]
            head += 1
            for a in range(4):
                for f in node_elems[conn[e, a]]:
                    if len(members) >= chunk_size:
                        break
                    if elem_chunk[f] < 0:
                        elem_chunk[f] = c
                        members.append(f)
                if len(members) >= chunk_size:
                    break
        chunks.append(members)
    chunk_color = [-1] * len(chunks)
    for c, members in enumerate(chunks):
        used = set()
        for e in members:
            for a in range(4):
                for f in node_elems[conn[e, a]]:
                    oc = elem_chunk[f]
                    if oc != c and chunk_color[oc] >= 0:
                        used.add(chunk_color[oc])
        col = 0
        while col in used:
            col += 1
        chunk_color[c] = col
    elem_color = [-1] * ne
    for c, members in enumerate(chunks):
        for k, e in enumerate(members):
            elem_color[e] = k
    stride = max_ec + 1
    emap = np.asarray(emap).reshape(-1, 16)
    tb, tn = {}, {}
    times = [chunk_color[elem_chunk[e]] * stride + elem_color[e] for e in range(ne)]
    for e in range(ne):
        t = times[e]
        for k in range(16):
            b = int(emap[e, k])
            tb[b] = min(tb.get(b, 1 << 30), t)
        for a in range(4):
            n = int(conn[e, a])
            tn[n] = min(tn.get(n, 1 << 30), t)
    ft = np.zeros(ne, np.uint32)
    for e in range(ne):
        t = times[e]
        m = 0
        for k in range(16):
            if tb[int(emap[e, k])] == t:
                m |= 1 << k
        for a in range(4):
            if tn[int(conn[e, a])] == t:
                m |= 1 << (16 + a)
        ft[e] = m
    return {"elem_chunk": np.array(elem_chunk, np.int32),
            "chunk_color": np.array(chunk_color, np.int32),
            "elem_color": np.array(elem_color, np.int32), "first_touch": ft,
            "num_chunk_colors": max(chunk_color) + 1, "num_chunks": len(chunks)}
