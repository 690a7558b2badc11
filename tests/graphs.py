"""Hand-made graphs with known answers, shared by CPU and GPU tests."""

import numpy as np


def from_edges(n, edges, weights=None):
    """CSR from a directed edge list, rows kept in the given order."""
    rows = [[] for _ in range(n)]
    for i, (u, v) in enumerate(edges):
        rows[u].append((v, None if weights is None else weights[i]))
    rs = np.zeros(n + 1, dtype=np.uint32)
    dst, w = [], []
    for u in range(n):
        rs[u + 1] = rs[u] + len(rows[u])
        for v, x in rows[u]:
            dst.append(v)
            w.append(x)
    dst = np.array(dst, dtype=np.uint32)
    wa = None if weights is None else np.array(w, dtype=np.int32)
    return rs, dst, wa


def undirected(n, pairs, weights=None):
    edges, ws = [], []
    for i, (u, v) in enumerate(pairs):
        edges += [(u, v), (v, u)]
        if weights is not None:
            ws += [weights[i], weights[i]]
    return from_edges(n, edges, ws if weights is not None else None)


def path(n, w=None):
    return undirected(n, [(i, i + 1) for i in range(n - 1)], None if w is None else [w] * (n - 1))


def star(n_leaves, w=None):
    """Hub 0 with n_leaves leaves: degree > CTA size hits the large-degree tiers."""
    return undirected(n_leaves + 1, [(0, i) for i in range(1, n_leaves + 1)],
                      None if w is None else [w + (i % 7) for i in range(n_leaves)])


def hand_cases():
    """(name, row_start, edge_dst, edge_data) for the edge cases the reference
    path meets: isolated source, disconnected parts, self loops, duplicate
    edges, zero-degree vertices, a hub above every degree threshold."""
    cases = []
    cases.append(("single",) + from_edges(1, [], []))
    cases.append(("path17",) + path(17, 3))
    cases.append(("star5000",) + star(5000, 2))
    cases.append(("disconnected",) + undirected(10, [(0, 1), (1, 2), (5, 6), (7, 8)], [4, 1, 2, 9]))
    cases.append(("selfloops_dups",) + from_edges(6, [(0, 0), (0, 1), (0, 1), (1, 2), (2, 2), (2, 3), (3, 0),
                                                      (1, 4), (4, 1), (4, 4)], [5, 3, 2, 7, 1, 1, 1, 9, 9, 1]))
    cases.append(("zero_degree_tail",) + from_edges(8, [(0, 3), (3, 5), (5, 0)], [1, 1, 1]))
    rng = np.random.default_rng(7)
    n = 3000
    pairs = [(int(a), int(b)) for a, b in rng.integers(0, n, size=(12000, 2))]
    cases.append(("random3000",) + undirected(n, pairs, [int(x) for x in rng.integers(1, 100, size=len(pairs))]))
    return cases
