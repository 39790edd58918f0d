"""Parity of the sm_100a path with the reference, through the C ABI.

Candidate sets, candidate-edge tables, matching orders, memory cost and
embedding counts must be identical (bit-exact integer results) to what the
reference computes: its recorded HPRD counts and the fixtures dumped from the
reference's own code (tests/golden), plus the oracle restatement on extra
cases."""
import os

import numpy as np
import pytest

from psm_benchmark_b200 import api
from oracle.oracle import OracleGraph
from tests import golden_data as gd
from tests.gpu_common import check_run_against_dump, engine  # noqa: F401

pytestmark = pytest.mark.gpu

METHODS = {"GQL_GQL": "GQL_GQL_GQL", "CFL_CFL": "CFL_CFL_EXPLORE", "NLF_GQL": "NLF_GQL_LFTJ"}


@pytest.fixture(scope="module")
def hprd_dev():
    g, qs, counts = gd.hprd()
    return api.DataGraph.from_graph(g), qs, counts


@pytest.mark.parametrize("qi", range(1, 11))
@pytest.mark.parametrize("m", list(METHODS))
def test_hprd(engine, hprd_dev, qi, m):
    dg, qs, counts = hprd_dev
    with api.Run(engine, dg, qs[qi - 1], METHODS[m]) as run:
        assert run.result.count == counts[qi - 1]
        assert run.result.status == 0
        check_run_against_dump(run, gd.golden()["hprd"]["dumps"][f"{qi}:{m}"])


@pytest.mark.parametrize("name", [n for n, _ in gd.synthetic_cases()])
def test_synthetic_against_reference(engine, name):
    case = dict(gd.synthetic_cases())[name]
    dg = api.DataGraph.from_graph(gd.synthetic_graph(name))
    for j, entry in enumerate(case["queries"]):
        q = gd.query_from_rec(entry["query"])
        for m, d in entry["methods"].items():
            with api.Run(engine, dg, q, m, cap=entry["cap"]) as run:
                assert run.result.count == d["count"], (name, j, m)
                check_run_against_dump(run, d)


def test_batch_equals_plain(engine):
    """Per-query counts of the batched path equal the plain path's."""
    name = "rmat12"
    case = dict(gd.synthetic_cases())[name]
    dg = api.DataGraph.from_graph(gd.synthetic_graph(name))
    qs = [gd.query_from_rec(e["query"]) for e in case["queries"]]
    caps = [e["cap"] for e in case["queries"]]
    for m in ("CFL_CFL_EXPLORE", "GQL_GQL_GQL"):
        plain = [api.match(engine, dg, q, m, cap=c).count for q, c in zip(qs, caps)]
        ref = [e["methods"][m]["count"] for e in case["queries"]]
        assert plain == ref
        # one batch per cap value (the cap is a per-launch option)
        for c in sorted(set(caps)):
            idx = [i for i, x in enumerate(caps) if x == c]
            batch = [r.count for r in api.match_batch(engine, dg, [qs[i] for i in idx], m, cap=c)]
            assert batch == [plain[i] for i in idx]


def test_embeddings_match_oracle(engine):
    """Full embedding sets of small queries."""
    g = gd.synthetic_graph("rmat12")
    og = OracleGraph(g)
    dg = api.DataGraph.from_graph(g)
    case = dict(gd.synthetic_cases())["rmat12"]
    checked = 0
    for entry in case["queries"]:
        q = gd.query_from_rec(entry["query"])
        ref = og.run(q, "CFL", "CFL", emit_limit=200000)
        if ref.count > 200000 or ref.count == 0:
            continue
        with api.Run(engine, dg, q, "CFL_CFL_EXPLORE", emit=ref.count + 10) as run:
            got = run.embeddings()
        assert got.shape[0] == ref.count
        assert set(map(tuple, got.tolist())) == set(map(tuple, ref.embeddings.tolist()))
        checked += 1
    assert checked >= 5


def test_edge_cases(engine):
    from psm_benchmark_b200.graphs import Graph
    g = gd.synthetic_graph("rmat12")
    og = OracleGraph(g)
    dg = api.DataGraph.from_graph(g)
    l0 = int(g.labels[0])
    cases = [
        Graph.from_edges(1, [l0], []),                              # single vertex
        Graph.from_edges(2, [l0, l0], [(0, 1)]),                    # one edge, same labels
        Graph.from_edges(3, [l0, 10**6, l0], [(0, 1), (1, 2)]),     # label absent from the data graph
        Graph.from_edges(4, [l0, l0, l0, l0], [(0, 1), (1, 2), (2, 3), (3, 0)]),
    ]
    for q in cases:
        for m in ("CFL_CFL_EXPLORE", "GQL_GQL_GQL"):
            f, o, _ = m.split("_")
            ref = og.run(q, f, o, cap=10**6, want_tables=False)
            got = api.match(engine, dg, q, m, cap=10**6)
            assert got.count == ref.count, (q.labels, m)


def test_cap_is_exact(engine):
    """With a cap the count is min(total, cap) exactly."""
    from psm_benchmark_b200.graphs import Graph
    g = gd.synthetic_graph("rmat12")
    dg = api.DataGraph.from_graph(g)
    l0 = int(g.labels[0])
    star = Graph.from_edges(4, [l0, l0, l0, l0], [(0, 1), (0, 2), (0, 3)])
    full = api.match(engine, dg, star, "CFL_CFL_EXPLORE").count
    assert full > 1000
    for cap in (1, 7, 999, full - 1, full, full + 5):
        assert api.match(engine, dg, star, "CFL_CFL_EXPLORE", cap=cap).count == min(full, cap)


def test_algorithmic_bytes_match_oracle(engine):
    """The enumerator's algorithmic bytes (the input volume of the
    reference's intersections: 8 B of row offsets + 4 B per entry of every
    backward-neighbour row, for every extended partial embedding) equal the
    oracle's instrumented count, with and without the enumerator's caches."""
    g, qs, counts = gd.hprd()
    og = OracleGraph(g)
    dg = api.DataGraph.from_graph(g)
    os.environ["PSM_ENUM_CACHE"] = "0"
    try:
        plain_engine = api.Engine(arena_bytes=1 << 30)
    finally:
        del os.environ["PSM_ENUM_CACHE"]
    try:
        for q in qs:
            for f, o, m in (("CFL", "CFL", "CFL_CFL_EXPLORE"), ("GQL", "GQL", "GQL_GQL_GQL")):
                ref = og.run(q, f, o, want_tables=False)
                for e in (engine, plain_engine):
                    got = api.match(e, dg, q, m)
                    assert got.count == ref.count
                    assert got.alg_bytes == int(ref.depth_bytes.sum()), (f, o)
    finally:
        plain_engine.close()
    # every plain_small query under both methods: these include orders whose
    # last two depths are counted through the weight memo
    syn = gd.synthetic_graph("plain_small")
    og = OracleGraph(syn)
    dg = api.DataGraph.from_graph(syn)
    case = dict(gd.synthetic_cases())["plain_small"]
    for entry in case["queries"]:
        q = gd.query_from_rec(entry["query"])
        for f, m in (("GQL", "GQL_GQL_GQL"), ("CFL", "CFL_CFL_EXPLORE")):
            ref = og.run(q, f, f, cap=entry["cap"], want_tables=False)
            got = api.match(engine, dg, q, m, cap=entry["cap"])
            assert got.count == ref.count
            if not entry["cap"] or ref.count < entry["cap"]:
                assert got.alg_bytes == int(ref.depth_bytes.sum()), (m, q.num_vertices)


def test_algorithmic_bytes_of_capped_queries(engine):
    """A capped query stops part-way through the search tree. Its bytes and
    its unclamped count (count_internal) come from the same extended partial
    embeddings, so: count_internal lies between the cap and the full count,
    and the bytes are at most the full tree's bytes (the oracle's exact
    figure), also after scaling them to the cap (bytes x cap / count_internal,
    the numerator of the bench's roofline)."""
    g, qs, counts = gd.hprd()
    og = OracleGraph(g)
    dg = api.DataGraph.from_graph(g)
    checked = 0
    for q in qs:
        full = og.run(q, "CFL", "CFL", want_tables=False)
        full_bytes = int(full.depth_bytes.sum())
        if full.count < 30:
            continue
        for cap in (full.count // 3, full.count - 1):
            got = api.match(engine, dg, q, "CFL_CFL_EXPLORE", cap=cap)
            assert got.count == cap
            assert cap <= got.count_internal <= full.count
            assert got.alg_bytes <= full_bytes
            assert got.alg_bytes * cap / got.count_internal <= full_bytes
            checked += 1
        got = api.match(engine, dg, q, "CFL_CFL_EXPLORE")
        assert got.count_internal == got.count == full.count
    assert checked >= 4
