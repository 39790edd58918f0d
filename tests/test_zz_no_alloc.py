"""The allocation-free recount entry point, psm_run_recount_noalloc.

It exists for callers that cannot allocate device memory when they need a
count (inside stream capture, allocation-free serving loops, hosts whose
device memory belongs to another runtime). The test calls it through the C
ABI on prepared runs and checks, for two calls in a row, that its count is
exactly the count of the ordinary entry point (integer counts: no
tolerance). This file is collected last so that a failure here never hides
the rest of the suite; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

from psm_benchmark_b200 import api, gen
from psm_benchmark_b200.graphs import Graph
from psm_benchmark_b200 import native as N
from tests import golden_data as gd

pytestmark = pytest.mark.gpu


def test_recount_noalloc_matches_plain_path():
    g = gd.synthetic_graph("rmat12")
    case = dict(gd.synthetic_cases())["rmat12"]
    queries = [gd.query_from_rec(e["query"]) for e in case["queries"][:8]]
    with api.Engine(arena_bytes=1 << 30) as eng:
        dg = api.DataGraph.from_graph(g)
        checked = 0
        for q in queries:
            for method, cap in (("CFL_CFL_EXPLORE", 0), ("GQL_GQL_GQL", 1000)):
                with api.Run(eng, dg, q, method, cap=cap) as run:
                    expected = run.result.count
                    for _ in range(2):  # two calls in a row share the static scratch
                        cnt = C.c_uint64(0)
                        over = C.c_uint32(1)
                        rc = N.lib().psm_run_recount_noalloc(run._h, cap, 60.0, C.byref(cnt), C.byref(over))
                        assert rc == N.PSM_OK, N.lib().psm_last_error()
                        assert over.value == 0
                        assert cnt.value == expected
                checked += 1
        dg.close()
    assert checked == 2 * len(queries)


def test_recount_noalloc_rejects_emit_runs():
    g = gd.synthetic_graph("rmat12")
    case = dict(gd.synthetic_cases())["rmat12"]
    q = gd.query_from_rec(case["queries"][0]["query"])
    with api.Engine(arena_bytes=1 << 30) as eng:
        dg = api.DataGraph.from_graph(g)
        with api.Run(eng, dg, q, "CFL_CFL_EXPLORE", emit=16) as run:
            cnt = C.c_uint64(0)
            rc = N.lib().psm_run_recount_noalloc(run._h, 0, 60.0, C.byref(cnt), None)
            assert rc == N.PSM_ERR_ARG
        dg.close()


def _kept_failed_run(dg, q):
    """A run whose preparation failed on the device (its candidate tables did
    not fit the arena) but whose handle psm_run_create kept. Found by
    bisecting the context's arena size between a size where the host-side
    setup already fails and one where the query runs."""
    qb = api._QueryBuf(q)
    # cap 1: a query that prepares successfully stops at its first embedding
    opt = api.options("CFL_CFL_EXPLORE", 1, 60.0, 0)
    lo, hi = 1 << 20, 1 << 30
    for _ in range(40):
        size = (lo + hi) // 2
        try:
            eng = api.Engine(arena_bytes=size)
        except N.PsmError:  # smaller than the context's fixed region
            lo = size
            continue
        h = C.c_void_p()
        res = N.Result()
        rc = N.lib().psm_run_create(eng._h, dg._h, C.byref(qb.desc), C.byref(opt), C.byref(h), C.byref(res))
        if rc == N.PSM_OK:
            N.lib().psm_run_free(h)
            eng.close()
            hi = size
        elif rc == N.PSM_ERR_OOM and not h.value:
            eng.close()
            lo = size
        else:
            assert rc == N.PSM_ERR_OOM, rc
            return eng, h
        if hi - lo <= 64:
            break
    pytest.fail("no arena size left the run's preparation out of memory")


def test_recount_noalloc_refuses_failed_preparation():
    # a star of six same-label leaves on a single-label graph: its candidate
    # tables (every candidate's whole row, per query edge and direction) are
    # large, which leaves a wide window of arena sizes where the host-side
    # setup fits but the tables do not
    g = gen.make_graph("rmat", 40, scale=11, edge_factor=8, num_labels=1)
    q = Graph.from_edges(7, np.zeros(7, np.uint32), [(0, i) for i in range(1, 7)])
    dg = api.DataGraph.from_graph(g)
    with api.Engine(arena_bytes=1 << 30) as big:
        assert api.match(big, dg, q, "CFL_CFL_EXPLORE", cap=1).table_entries * 4 > 1 << 20
    eng, h = _kept_failed_run(dg, q)
    try:
        cnt = C.c_uint64(7)
        rc = N.lib().psm_run_recount_noalloc(h, 0, 60.0, C.byref(cnt), None)
        assert rc == N.PSM_ERR_OOM, N.lib().psm_last_error()
        assert cnt.value == 7  # nothing written on refusal
    finally:
        N.lib().psm_run_free(h)
        eng.close()
        dg.close()
