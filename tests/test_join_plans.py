"""Decomposition patterns and join plans of the join path (host only).

The reference's -Qpattern values (utility/splitGraph/SplitGraph.cpp: STAR,
TWINTWIG, SEED, SKETCHTREE) and this library's BOUNDED and COST patterns,
left-deep or bushy (-JoinMethod LEFTDEEP / BUSHY). Every plan must be a
valid decomposition: each query edge inside some unit, each unit connected,
each join between partial results that share a query vertex, each unit and
each join result used exactly once, and the shapes of the pattern (twin-twigs
of at most three vertices, stars, root-to-leaf paths, the unit bound).
"""
import numpy as np
import pytest

from psm_benchmark_b200 import api, gen
from psm_benchmark_b200.graphs import Graph
from tests import golden_data as gd


def bits(m):
    return [i for i in range(32) if (m >> i) & 1]


def connected(q, mask):
    vs = bits(mask)
    seen = {vs[0]}
    stack = [vs[0]]
    while stack:
        u = stack.pop()
        for v in q.neighbors(u):
            v = int(v)
            if (mask >> v) & 1 and v not in seen:
                seen.add(v)
                stack.append(v)
    return len(seen) == len(vs)


def check_plan(q, units, joins):
    n = q.num_vertices
    for a, b in q.edge_list():
        assert any((m >> int(a)) & 1 and (m >> int(b)) & 1 for m in units), (a, b)
    for m in units:
        assert connected(q, m)
    U = len(units)
    masks = list(units)
    used = [0] * (U + len(joins))
    for j, (a, b) in enumerate(joins):
        assert a < U + j and b < U + j
        used[a] += 1
        used[b] += 1
        assert masks[a] & masks[b], "a join without a shared query vertex"
        masks.append(masks[a] | masks[b])
    # every unit and every result but the last is consumed exactly once
    assert all(c == 1 for c in used[:-1]) if joins else U == 1
    assert masks[-1] == (1 << n) - 1


def queries():
    g, hq, _ = gd.hprd()
    qs = list(hq)
    rg = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    qs += gen.make_queries(rg, [8, 12, 16, 20, 24, 28, 32] * 2, gen.BASE_SEED + 77)
    # a cycle, a clique and a long path
    qs.append(Graph.from_edges(6, np.zeros(6, np.uint32), [(i, (i + 1) % 6) for i in range(6)]))
    qs.append(Graph.from_edges(6, np.zeros(6, np.uint32), [(a, b) for a in range(6) for b in range(a + 1, 6)]))
    qs.append(Graph.from_edges(10, np.zeros(10, np.uint32), [(i, i + 1) for i in range(9)]))
    return qs


@pytest.mark.parametrize("pattern", ["BOUNDED", "STAR", "TWINTWIG", "SEED", "SKETCHTREE", "COST"])
@pytest.mark.parametrize("join_method", ["LEFTDEEP", "BUSHY"])
def test_plans_are_valid(pattern, join_method):
    checked = 0
    for q in queries():
        try:
            units, joins = api.join_plan(q, pattern, join_method, max_unit_vertices=6)
        except Exception as e:  # more units than the result record holds
            assert "units" in str(e), e
            continue
        check_plan(q, units, joins)
        sizes = [len(bits(m)) for m in units]
        if pattern == "TWINTWIG" or pattern == "SEED":
            assert max(sizes) <= 3
        if pattern in ("BOUNDED", "COST"):
            assert max(sizes) <= 6
        if pattern == "STAR":
            # a centre adjacent to every other unit vertex
            for m in units:
                vs = bits(m)
                assert any(all(w == c or q.neighbors(c).tolist().count(w) for w in vs) for c in vs)
        if pattern == "SKETCHTREE":
            # every unit holds the root (the vertex of highest degree)
            deg = np.diff(q.off.astype(np.int64))
            root = int(np.argmax(deg))
            assert all((m >> root) & 1 for m in units)
        if join_method == "LEFTDEEP" and pattern != "SKETCHTREE":
            # a chain: each join takes the previous result
            for j, (a, b) in enumerate(joins[1:], start=1):
                assert a == len(units) + j - 1
        checked += 1
    assert checked >= 20


def test_sketch_tree_joins_along_the_tree():
    # a spider: three legs of two vertices around vertex 0
    q = Graph.from_edges(7, np.zeros(7, np.uint32), [(0, 1), (1, 2), (0, 3), (3, 4), (0, 5), (5, 6)])
    units, joins = api.join_plan(q, "SKETCHTREE")
    assert sorted(units) == sorted([0b0000111, 0b0011001, 0b1100001])
    assert len(joins) == 2


def test_cost_plans_respect_the_unit_bound():
    """COST searches the bounded decompositions of every start vertex and
    unit bounds max_unit .. max_unit - 4: its plans stay valid and bounded."""
    rg = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    for q in gen.make_queries(rg, [16, 20, 24], gen.BASE_SEED + 78):
        for jm in ("LEFTDEEP", "BUSHY"):
            u_c, j_c = api.join_plan(q, "COST", jm, max_unit_vertices=8)
            check_plan(q, u_c, j_c)
            assert max(len(bits(m)) for m in u_c) <= 8
