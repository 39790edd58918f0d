"""The time limit of a query (the reference's -time_limit: TaskPool::
checkOverTime, matching/TaskPool.cpp:198-205, sets `overtime` and the log
block prints 'Overtime: 1', matching/StudyPerformance.cpp:1717-1781).

A star with k leaves on a single-label graph without self loops has exactly
sum_v deg(v)! / (deg(v) - k)! embeddings (the leaves are distinct neighbours
of the centre), so the true count is known without enumerating it. With k = 6
on an R-MAT graph that count is far beyond what the GPU enumerates in the
time limits used here, so the limit must end the query: the library returns
PSM_ERR_TIMEOUT with overtime = 1 and a partial count no larger than the true
one, promptly, and the context serves the next query with an exact count.
"""
import time
from math import perm

import numpy as np
import pytest

from psm_benchmark_b200 import api, gen
from psm_benchmark_b200.graphs import Graph
from psm_benchmark_b200.native import PSM_ERR_TIMEOUT, PSM_OK

pytestmark = pytest.mark.gpu


def star(k: int) -> Graph:
    return Graph.from_edges(k + 1, np.zeros(k + 1, np.uint32), [(0, i) for i in range(1, k + 1)])


def star_count(g: Graph, k: int) -> int:
    return sum(perm(int(d), k) for d in np.diff(g.off.astype(np.int64)) if d >= k)


@pytest.fixture(scope="module")
def one_label_graph():
    return gen.make_graph("rmat", 40, scale=11, edge_factor=8, num_labels=1)


def test_time_limit_ends_query_and_context_stays_usable(one_label_graph):
    g = one_label_graph
    big = star_count(g, 6)
    assert big > 10**15  # far beyond what 50 ms of enumeration can reach
    with api.Engine(arena_bytes=1 << 30) as eng:
        dg = api.DataGraph.from_graph(g)
        for method in ("CFL_CFL_EXPLORE", "GQL_GQL_GQL"):
            t = time.perf_counter()
            r = api.match(eng, dg, star(6), method, cap=0, time_limit=0.05)
            wall = time.perf_counter() - t
            assert r.status == PSM_ERR_TIMEOUT
            assert r.overtime == 1
            assert 0 < r.count < big
            assert wall < 2.0, wall
            # the next query on the same context runs to its exact count
            r3 = api.match(eng, dg, star(3), method, cap=0, time_limit=60.0)
            assert r3.status == PSM_OK and r3.overtime == 0
            assert r3.count == star_count(g, 3)
        # a cap below the partial count still clamps a timed-out query
        r = api.match(eng, dg, star(6), "CFL_CFL_EXPLORE", cap=1000, time_limit=0.05)
        assert r.count == 1000 and r.overtime == 0 and r.status == PSM_OK
        dg.close()


def test_time_limit_in_batch_ends_only_the_slow_query(one_label_graph):
    g = one_label_graph
    with api.Engine(arena_bytes=1 << 30) as eng:
        dg = api.DataGraph.from_graph(g)
        res = api.match_batch(eng, dg, [star(3), star(6), star(2)], "CFL_CFL_EXPLORE", cap=0, time_limit=0.1)
        assert res[1].overtime == 1 and res[1].count < star_count(g, 6)
        # queries that finish inside the limit keep their exact counts
        for r, k in ((res[0], 3), (res[2], 2)):
            if not r.overtime:
                assert r.count == star_count(g, k)
        r = api.match(eng, dg, star(2), "CFL_CFL_EXPLORE", cap=0, time_limit=60.0)
        assert r.status == PSM_OK and r.count == star_count(g, 2)
        dg.close()
