"""Serving runtime: continuous batching over a resident graph.

Each request's count in the mix (several lanes running batches side by side,
requests arriving while others are on the GPU) equals its count alone
(psm_match); requests whose estimated device memory exceeds a lane's budget
are refused with PSM_ERR_OOM instead of being run.
"""
import threading
import time

import numpy as np
import pytest

from psm_benchmark_b200 import api, gen
from psm_benchmark_b200.native import PSM_ERR_OOM, PSM_OK
from tests import golden_data as gd
from tests.gpu_common import engine  # noqa: F401

pytestmark = pytest.mark.gpu


def mixed_queries():
    g = gd.synthetic_graph("rmat12")
    sizes = [4, 6, 8, 12, 16] * 8
    return g, gen.make_queries(g, sizes, gen.BASE_SEED + 9)


def test_results_alone_equal_results_in_the_mix(engine):
    g, qs = mixed_queries()
    dg = api.DataGraph.from_graph(g)
    cap = 10**6
    alone = [api.match(engine, dg, q, "CFL_CFL_EXPLORE", cap=cap, time_limit=60).count for q in qs]
    with api.Server(dg, "CFL_CFL_EXPLORE", cap=cap, time_limit=60, lanes=3, max_batch=6,
                    lane_arena_bytes=1 << 30) as srv:
        tickets = {}
        rng = np.random.default_rng(3)

        def producer():
            # bursts of arrivals spread over the run: some requests queue up
            # behind running batches and are admitted together
            for i, q in enumerate(qs):
                tickets[srv.submit(q)] = i
                if i % 8 == 7:
                    time.sleep(float(rng.uniform(0, 0.004)))

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        res = srv.drain(len(qs), timeout_s=300)
    assert len(res) == len(qs)
    for r in res:
        assert r.status == PSM_OK
        assert r.count == alone[tickets[r.ticket]], tickets[r.ticket]
        assert r.submit_ns <= r.start_ns <= r.done_ns
    # continuous batching: several lanes' batches were on the GPU at once,
    # and some requests were batched together
    spans = sorted({(r.lane, r.start_ns, r.done_ns) for r in res}, key=lambda x: x[1])
    overlap = any(a[0] != b[0] and b[1] < a[2] for i, a in enumerate(spans) for b in spans[i + 1:])
    assert overlap
    assert max(r.batch_size for r in res) > 1


def test_admission_refuses_requests_beyond_the_budget(engine):
    # one label: every candidate bucket is the whole graph
    g0 = gen.make_graph("rmat", 6, scale=16, edge_factor=8, num_labels=1)
    qs = gen.make_queries(g0, [3, 12], gen.BASE_SEED + 11)
    dg = api.DataGraph.from_graph(g0)
    with api.Server(dg, "GQL_GQL_GQL", cap=1000, time_limit=60, lanes=1, max_batch=4,
                    lane_arena_bytes=64 << 20) as srv:
        small, budget = srv.estimate(qs[0])
        big, _ = srv.estimate(qs[1])
        assert small <= budget < big
        t_small = srv.submit(qs[0])
        t_big = srv.submit(qs[1])
        res = {r.ticket: r for r in srv.drain(2, timeout_s=120)}
    assert res[t_big].status == PSM_ERR_OOM
    assert res[t_small].status == PSM_OK
    assert res[t_small].count == api.match(engine, dg, qs[0], "GQL_GQL_GQL", cap=1000).count


def test_server_tuning_reaches_every_lane_and_keeps_counts(engine):
    """psm_server_set_batch_tuning: the lanes take the setting before their
    next batch; counts do not change. Out-of-range settings are refused."""
    from psm_benchmark_b200.native import PsmError
    g, qs = mixed_queries()
    dg = api.DataGraph.from_graph(g)
    cap = 10**6
    alone = [api.match(engine, dg, q, "CFL_CFL_EXPLORE", cap=cap, time_limit=60).count for q in qs]
    with api.Server(dg, "CFL_CFL_EXPLORE", cap=cap, time_limit=60, lanes=2, max_batch=8,
                    lane_arena_bytes=1 << 30) as srv:
        with pytest.raises(PsmError):
            srv.set_batch_tuning("BLOCK", 0, 4, "AUTO")
        for setting in (("BLOCK", 2, 2, "MERGE"), ("BLOCK", 32, 4, "BINARY"), ("RULE", 8, 4, "AUTO")):
            srv.set_batch_tuning(*setting)
            tickets = {srv.submit(q): i for i, q in enumerate(qs)}
            res = srv.drain(len(qs), timeout_s=300)
            assert len(res) == len(qs)
            for r in res:
                assert r.status == PSM_OK
                assert r.count == alone[tickets[r.ticket]], (setting, tickets[r.ticket])
