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
