"""ORACLE -- TEST INFRASTRUCTURE ONLY.

CPU restatement of the reference's hash join of partial-embedding relations
and checks of a query decomposition. Only tests import this module, as the
checker; the product path never calls it.

hash_join restates JoinCollect::concateTwoTabels (matching/JoinCollect.cpp:
60-153) with NoPartitionHashJoin (utility/hashjoin/hashjoin.cpp:337-572
execute, :591-779 constructRow):
  - join keys: query vertices present in both relations (:74-114);
  - R is hashed on its key columns, every S row probes it (:337-420);
  - for a key match, the output row is S's columns followed by R's non-key
    columns, and it is kept only if none of R's non-key values occurs among
    S's values (the visited[] test of constructRow, :598-725).
The reference tests R's values against all of S's; two columns can hold the
same data vertex only if their query vertices share a label, so with
`vertex_label` given the test is restricted to same-label columns, which
gives the same rows.
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np


def hash_join(R, r_vertex, S, s_vertex, vertex_label=None):
    """Returns (rows as a list of tuples, out_vertex)."""
    r_vertex = [int(x) for x in r_vertex]
    s_vertex = [int(x) for x in s_vertex]
    keys = [v for v in r_vertex if v in s_vertex]
    rk = [r_vertex.index(v) for v in keys]
    sk = [s_vertex.index(v) for v in keys]
    rx = [i for i, v in enumerate(r_vertex) if v not in keys]
    table = defaultdict(list)
    for row in np.asarray(R, dtype=np.int64).reshape(-1, len(r_vertex)):
        table[tuple(int(row[i]) for i in rk)].append(row)
    out = []
    for srow in np.asarray(S, dtype=np.int64).reshape(-1, len(s_vertex)):
        key = tuple(int(srow[i]) for i in sk)
        for rrow in table.get(key, ()):
            ok = True
            for i in rx:
                for j, sv in enumerate(s_vertex):
                    if vertex_label is not None and vertex_label[sv] != vertex_label[r_vertex[i]]:
                        continue
                    if int(srow[j]) == int(rrow[i]):
                        ok = False
            if ok:
                out.append(tuple(int(x) for x in srow) + tuple(int(rrow[i]) for i in rx))
    return out, s_vertex + [r_vertex[i] for i in rx]


def check_decomposition(n, edges, unit_masks, max_unit):
    """Raises AssertionError unless the units cover every vertex and edge,
    stay within max_unit vertices, are connected, and each unit after the
    first shares a vertex with the units before it (so a left-deep join in
    unit order has a key at every step)."""
    edges = [(int(a), int(b)) for a, b in edges]
    unit_masks = [int(m) for m in unit_masks]
    adj = [0] * n
    for a, b in edges:
        adj[a] |= 1 << b
        adj[b] |= 1 << a
    covered_v = 0
    for k, m in enumerate(unit_masks):
        assert bin(m).count("1") <= max_unit or n == 1, (k, m)
        assert m and m < (1 << n)
        # connected inside the unit
        start = m & -m
        comp = start
        while True:
            grow = comp
            x = comp
            while x:
                low = x & -x
                grow |= adj[low.bit_length() - 1] & m
                x ^= low
            if grow == comp:
                break
            comp = grow
        assert comp == m, ("unit not connected", k, m)
        if k > 0:
            assert m & covered_v, ("no join key", k)
        covered_v |= m
    assert covered_v == (1 << n) - 1, "vertex not covered"
    for a, b in edges:
        assert any((m >> a) & 1 and (m >> b) & 1 for m in unit_masks), ("edge not covered", a, b)
