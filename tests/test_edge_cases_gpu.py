"""Edge cases of the matching path through the C ABI: the largest query
size (32 vertices), degenerate data graphs, and queries that cannot match.
Counts are compared with the oracle restatement."""
import numpy as np
import pytest

from oracle.oracle import OracleGraph
from psm_benchmark_b200 import api, gen
from psm_benchmark_b200.graphs import Graph
from psm_benchmark_b200.native import PsmError
from tests import golden_data as gd
from tests.gpu_common import engine  # noqa: F401

pytestmark = pytest.mark.gpu


def test_largest_queries_match_oracle(engine):
    """32-vertex queries (the engine's maximum), sparse and dense, under both
    methods and in the batched path."""
    g = gd.synthetic_graph("rmat12")
    og = OracleGraph(g)
    dg = api.DataGraph.from_graph(g)
    qs = gen.make_queries(g, [32, 32, 32, 32], gen.BASE_SEED + 21)
    cap = 20000
    for f, m in (("CFL", "CFL_CFL_EXPLORE"), ("GQL", "GQL_GQL_GQL")):
        ref = [og.run(q, f, f, cap=cap, want_tables=False).count for q in qs]
        assert [api.match(engine, dg, q, m, cap=cap).count for q in qs] == ref
        assert [r.count for r in api.match_batch(engine, dg, qs, m, cap=cap)] == ref


def test_query_above_the_maximum_is_rejected(engine):
    g = gd.synthetic_graph("rmat12")
    dg = api.DataGraph.from_graph(g)
    n = 33
    q = Graph.from_edges(n, np.zeros(n, np.uint32), [(i, i + 1) for i in range(n - 1)])
    with pytest.raises(PsmError):
        api.match(engine, dg, q, "CFL_CFL_EXPLORE")


def tiny_graph(edges, labels):
    n = len(labels)
    return Graph.from_edges(n, np.asarray(labels, np.uint32), edges)


@pytest.mark.parametrize("method", ["CFL_CFL_EXPLORE", "GQL_GQL_GQL", "NLF_GQL_LFTJ"])
def test_degenerate_graphs(engine, method):
    f, o, _ = method.split("_")
    cases = []
    # a data graph without edges: an edge query has no match, a vertex query
    # matches every vertex of its label
    g0 = tiny_graph([], [0, 1, 0, 2, 0])
    cases.append((g0, tiny_graph([(0, 1)], [0, 0])))
    cases.append((g0, tiny_graph([], [0])))
    # a query with more vertices than the data graph
    g1 = tiny_graph([(0, 1), (1, 2)], [0, 0, 0])
    cases.append((g1, tiny_graph([(0, 1), (1, 2), (2, 3)], [0, 0, 0, 0])))
    # a triangle of one label in a 4-clique: 4 * 3 * 2 embeddings
    g2 = tiny_graph([(a, b) for a in range(4) for b in range(a + 1, 4)], [5, 5, 5, 5])
    cases.append((g2, tiny_graph([(0, 1), (1, 2), (0, 2)], [5, 5, 5])))
    # a query label the data graph does not carry
    cases.append((g2, tiny_graph([(0, 1)], [5, 9])))
    for g, q in cases:
        want = OracleGraph(g).run(q, f, o, want_tables=False).count
        dg = api.DataGraph.from_graph(g)
        assert api.match(engine, dg, q, method).count == want, (g.num_vertices, q.num_vertices)
        assert api.match_batch(engine, dg, [q, q], method)[1].count == want
    assert api.match(engine, api.DataGraph.from_graph(g2), cases[3][1], method).count == 24


def hub_graph():
    """6,000 vertices, 6 labels, sparse random edges plus hub rows that put
    label runs where row searches have their boundaries: one vertex adjacent
    to all others (runs of about 1,000 entries), one whose whole row is one
    label, one with runs of exactly 8 and 9 entries, and one adjacent only to
    the last label."""
    rng = np.random.default_rng(2024)
    V, L = 6000, 6
    lab = rng.integers(0, L, size=V).astype(np.uint32)
    lab[:4] = [0, 1, 2, 3]
    edges = set()
    for v in range(1, V):
        edges.add((0, v))
    for v in np.flatnonzero(lab == 0):
        if v > 3:
            edges.add((1, int(v)))
    for l, k in ((1, 8), (2, 9), (4, 1)):
        for v in np.flatnonzero(lab == l)[:k + 4][-k:]:
            if v > 3:
                edges.add((2, int(v)))
    for v in np.flatnonzero(lab == L - 1):
        if v > 3:
            edges.add((3, int(v)))
    while len(edges) < 6000 + 20000:
        a, b = (int(x) for x in rng.integers(4, V, size=2))
        if a != b:
            edges.add((min(a, b), max(a, b)))
    return Graph.from_edges(V, lab, sorted(edges))


def oracle_dump(r):
    return {"cands": r.candidates, "tables": [(a, b, off, adj) for (a, b), (off, adj) in r.tables.items()],
            "memory": r.memory_bytes, "order": list(r.order), "pivot": list(r.pivot)}


def test_hub_rows_match_oracle(engine):
    """Candidates, tables, orders and counts on hub rows (label runs of one
    to thousands of entries, at the start, middle and end of a row) equal the
    oracle's, under both methods."""
    from tests.gpu_common import check_run_against_dump
    g = hub_graph()
    og = OracleGraph(g)
    dg = api.DataGraph.from_graph(g)
    qs = [Graph.from_edges(4, [0, 1, 2, 5], [(0, 1), (0, 2), (0, 3)]),          # star on the all-adjacent hub
          Graph.from_edges(3, [1, 0, 0], [(0, 1), (0, 2)]),                     # the single-run row
          Graph.from_edges(3, [2, 1, 2], [(0, 1), (0, 2), (1, 2)]),             # the 8 / 9-entry runs
          Graph.from_edges(4, [3, 5, 5, 0], [(0, 1), (0, 2), (1, 3), (2, 3)])]  # the last label's run
    qs += gen.make_queries(g, [3, 4, 5, 6, 8], gen.BASE_SEED + 31)
    checked = 0
    for q in qs:
        for f, m in (("CFL", "CFL_CFL_EXPLORE"), ("GQL", "GQL_GQL_GQL")):
            ref = og.run(q, f, f, cap=10**6)
            with api.Run(engine, dg, q, m, cap=10**6) as run:
                check_run_against_dump(run, oracle_dump(ref))
                assert run.result.count == ref.count, (q.labels, m)
            checked += 1
    assert checked == 2 * len(qs)


def with_self_loops(g, every=8):
    """g with a self loop (v once in its own row) at every `every`-th vertex."""
    V = g.num_vertices
    rows = [list(g.neighbors(v)) for v in range(V)]
    for v in range(0, V, every):
        rows[v] = sorted(rows[v] + [v])
    off = np.zeros(V + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    nbr = np.array([w for r in rows for w in r], np.uint32)
    return Graph(off, nbr, np.asarray(g.labels, np.uint32))


def test_self_loops_in_the_data_graph(engine):
    """Self loops in the data graph: a vertex then sits in its own table rows
    and passes filters it would fail without the loop, but no injective
    embedding uses a loop. Counts equal the oracle's on the same graph and the
    counts without the loops, plain and batched. Eight labels make
    consecutive same-label depths common, where the enumerator's loop-free
    shortcuts would otherwise apply; about half the queries finish below the
    cap."""
    base = gd.synthetic_graph("rmat12")
    g0 = Graph(base.off, base.nbr, (np.asarray(base.labels) % 8).astype(np.uint32))
    g1 = with_self_loops(g0)
    og = OracleGraph(g1)
    d0, d1 = api.DataGraph.from_graph(g0), api.DataGraph.from_graph(g1)
    qs = gen.make_queries(g0, [4, 5, 6, 7, 8] * 3, gen.BASE_SEED + 41)
    cap = 2000000
    for f, m in (("CFL", "CFL_CFL_EXPLORE"), ("GQL", "GQL_GQL_GQL")):
        want = [og.run(q, f, f, cap=cap, want_tables=False).count for q in qs]
        assert [api.match(engine, d1, q, m, cap=cap).count for q in qs] == want
        assert [api.match(engine, d0, q, m, cap=cap).count for q in qs] == want
        assert [r.count for r in api.match_batch(engine, d1, qs, m, cap=cap)] == want
