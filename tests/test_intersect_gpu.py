"""Intersection variants of the enumerator (psm_batch_tuning.intersect).

The reference intersects by galloping for skewed pairs and by a merge for
balanced ones (utility/computesetintersection.cpp:5-30); the device has a warp
merge path, a lane two-cursor merge, a lane search that shrinks its range, the
chunked binary search and the bitmaps. Variants change the work, never the
counts:
  * the primitives themselves (psm_intersect_check, one warp) against numpy on
    empty, tiny, skewed, balanced and multi-tile arrays, with and without the
    output list and its cap;
  * every variant (AUTO, BINARY, MERGE), with and without the enumerator's
    caches, counts the reference's embeddings on HPRD and on the R-MAT
    fixtures, and the oracle's on a graph whose candidate sets are too large
    for the cache bitmaps (so the list intersections carry the work).
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle.oracle import OracleGraph
from psm_benchmark_b200 import api, gen
from psm_benchmark_b200 import native as N
from psm_benchmark_b200.graphs import Graph
from tests import golden_data as gd

pytestmark = pytest.mark.gpu

VARIANTS = ("AUTO", "BINARY", "MERGE")


def device_intersect(a, b, cap, filt):
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    counts = np.zeros(5, np.uint32)
    out = np.zeros(max(cap, 1), np.uint32)
    p = lambda x: x.ctypes.data_as(C.POINTER(C.c_uint32))  # noqa: E731
    N.check(N.lib().psm_intersect_check(p(a), len(a), p(b), len(b), cap, int(filt), p(counts), p(out)))
    return counts, out[: counts[3]]


def sorted_unique(rng, n, hi):
    return np.sort(rng.choice(hi, size=n, replace=False)).astype(np.uint32)


CASES = [(0, 0, 10), (0, 7, 10), (7, 0, 10), (1, 1, 1), (1, 1, 2), (31, 33, 64), (32, 32, 40), (33, 31, 200),
         (100, 3000, 4000), (3000, 100, 4000), (4096, 4096, 5000), (4096, 4097, 9000), (5000, 5000, 10**6),
         (8000, 8000, 9000), (20000, 7, 40000), (12000, 12000, 13000), (1, 9000, 9001)]


@pytest.mark.parametrize("na,nb,hi", CASES)
def test_primitives_match_numpy(na, nb, hi):
    rng = np.random.default_rng(na * 7919 + nb * 31 + hi)
    a, b = sorted_unique(rng, na, hi), sorted_unique(rng, nb, hi)
    common = np.intersect1d(a, b)
    kept = common[common % 3 != 0]
    for filt, want in ((False, common), (True, kept)):
        counts, out = device_intersect(a, b, cap=len(common) + 5, filt=filt)
        assert counts[0] == len(want)
        assert counts[1] == counts[2] == len(common)
        assert counts[4] == 0
        assert np.array_equal(out, want)
    if len(common) > 1:
        # an output that does not fit is refused, never written past the cap
        counts, _ = device_intersect(a, b, cap=len(common) - 1, filt=False)
        assert counts[4] == 1 and counts[3] <= len(common) - 1


def test_primitives_on_identical_and_disjoint_arrays():
    x = np.arange(0, 20000, 2, dtype=np.uint32)
    counts, out = device_intersect(x, x, cap=len(x), filt=False)
    assert list(counts[:4]) == [len(x)] * 4 and np.array_equal(out, x)
    counts, out = device_intersect(x, x + 1, cap=16, filt=False)
    assert list(counts[:4]) == [0, 0, 0, 0] and counts[4] == 0


def engine_with(intersect, cache=True):
    if not cache:
        os.environ["PSM_ENUM_CACHE"] = "0"
    try:
        eng = api.Engine(arena_bytes=2 << 30)
    finally:
        os.environ.pop("PSM_ENUM_CACHE", None)
    eng.set_batch_tuning(intersect=intersect)
    return eng


@pytest.mark.parametrize("intersect", VARIANTS)
@pytest.mark.parametrize("cache", [True, False])
def test_variants_count_the_reference_embeddings(intersect, cache):
    g, qs, counts = gd.hprd()
    with engine_with(intersect, cache) as eng:
        assert eng.batch_tuning()["intersect"] == intersect
        dg = api.DataGraph.from_graph(g)
        for m in ("CFL_CFL_EXPLORE", "GQL_GQL_GQL"):
            assert [api.match(eng, dg, q, m).count for q in qs] == list(counts)
        dg.close()
        for name, case in gd.synthetic_cases():
            dg = api.DataGraph.from_graph(gd.synthetic_graph(name))
            for e in case["queries"]:
                q = gd.query_from_rec(e["query"])
                for m, d in e["methods"].items():
                    assert api.match(eng, dg, q, m, cap=e["cap"]).count == d["count"], (name, m)
            dg.close()


def one_label(k, edges):
    return Graph.from_edges(k, np.zeros(k, np.uint32), edges)


@pytest.fixture(scope="module")
def wide_graph():
    """R-MAT scale 18, edge factor 2, one label: candidate sets of 37-62 K
    vertices, beyond the 32 K positions a cache bitmap covers."""
    return gen.make_graph("rmat", 7, scale=18, edge_factor=2, num_labels=1)


def test_variants_agree_beyond_the_bitmaps(wide_graph):
    g = wide_graph
    og = OracleGraph(g)
    clique = lambda k: one_label(k, [(a, b) for a in range(k) for b in range(a + 1, k)])  # noqa: E731
    exact = {"triangle": clique(3), "4-clique": clique(4)}
    want = {name: og.run(q, "CFL", "CFL", want_tables=False).count for name, q in exact.items()}
    assert want["triangle"] > 10**6 and want["4-clique"] > 10**7
    more = [clique(5), one_label(4, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2)]),
            one_label(5, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (1, 4)])]
    more += gen.make_queries(g, [5, 6, 8], gen.BASE_SEED + 303)
    seen = None
    for intersect in VARIANTS:
        for cache in (True, False):
            with engine_with(intersect, cache) as eng:
                dg = api.DataGraph.from_graph(g)
                for m in ("CFL_CFL_EXPLORE", "GQL_GQL_GQL"):
                    for name, q in exact.items():
                        r = api.match(eng, dg, q, m, time_limit=60)
                        assert not r.overtime and r.count == want[name], (intersect, cache, m, name)
                got = []
                for q in more:
                    r = api.match(eng, dg, q, "CFL_CFL_EXPLORE", cap=10**10, time_limit=60)
                    assert not r.overtime
                    got.append(r.count)
                dg.close()
            if seen is None:
                seen = got
            assert got == seen, (intersect, cache)
