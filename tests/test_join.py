"""Decomposition + hash-join path (the reference's -QorCandi Q mode).

CPU: the decomposition's structural guarantees on seeded queries, and the
join oracle against a nested-loop join. GPU: the device hash join against
the oracle (duplicates, multi-column keys, injectivity rejections, empty
sides), and psm_match_join against the reference's own Q-mode counts
(tests/golden/join_ref.json, made by tests/golden/make_join_golden.py) and
its recorded HPRD counts.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from psm_benchmark_b200 import api, gen
from psm_benchmark_b200.native import PsmError
from oracle.join_oracle import check_decomposition, hash_join
from tests import golden_data as gd
from tests.gpu_common import engine  # noqa: F401

JOIN_REF = Path(__file__).resolve().parent / "golden" / "join_ref.json"


def join_ref():
    return json.loads(JOIN_REF.read_text())


def some_queries():
    g = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    sizes = [4, 6, 8, 12, 16, 20, 24, 28, 32] * 2
    return gen.make_queries(g, sizes, gen.BASE_SEED + 7)


@pytest.mark.parametrize("max_unit", [2, 3, 4, 6, 12])
def test_decomposition_properties(max_unit):
    checked = 0
    for q in some_queries() + gd.hprd()[1]:
        try:
            masks = api.decompose(q, max_unit)
        except PsmError as e:
            # small units on a large dense query: more than PSM_MAX_UNITS units
            assert "units" in str(e) and q.num_edges > 32
            continue
        check_decomposition(q.num_vertices, [tuple(e) for e in q.edge_list()], masks, max_unit)
        checked += 1
    assert checked >= 10


def test_decomposition_sizes_for_large_queries():
    """24-32 vertex queries split into a few units of <= 12 vertices."""
    for q in some_queries():
        if q.num_vertices >= 24:
            masks = api.decompose(q, 12)
            assert 2 <= len(masks) <= 8, (q.num_vertices, len(masks))


def test_join_oracle_matches_nested_loops():
    rng = np.random.default_rng(5)
    for trial in range(20):
        R = rng.integers(0, 6, size=(rng.integers(0, 30), 3))
        S = rng.integers(0, 6, size=(rng.integers(0, 30), 3))
        rv, sv = [0, 1, 2], [2, 3, 1] if trial % 2 else [4, 3, 0]
        lab = [0, 1, 0, 1, 0]
        got, ov = hash_join(R, rv, S, sv, lab)
        want = []
        keys = [v for v in rv if v in sv]
        for s in S:
            for r in R:
                if any(r[rv.index(v)] != s[sv.index(v)] for v in keys):
                    continue
                rx = [i for i, v in enumerate(rv) if v not in keys]
                if any(lab[sv[j]] == lab[rv[i]] and s[j] == r[i] for i in rx for j in range(len(sv))):
                    continue
                want.append(tuple(int(x) for x in s) + tuple(int(r[i]) for i in rx))
        assert sorted(got) == sorted(want)
        assert ov == sv + [v for v in rv if v not in keys]


@pytest.mark.gpu
def test_device_hash_join_matches_oracle(engine):
    rng = np.random.default_rng(11)
    cases = []
    # heavy duplicates on a single key column, same labels everywhere
    cases.append((rng.integers(0, 8, size=(500, 3)), [0, 1, 2], rng.integers(0, 8, size=(400, 3)), [2, 3, 4], None))
    # three key columns, labels restrict the injectivity test
    cases.append((rng.integers(0, 5, size=(2000, 5)), [0, 1, 2, 3, 4], rng.integers(0, 5, size=(1500, 4)),
                  [1, 3, 4, 6], [0, 1, 0, 1, 0, 1, 0]))
    # no key value in common
    cases.append((rng.integers(0, 10, size=(100, 2)), [0, 1], rng.integers(20, 30, size=(100, 2)), [1, 2], None))
    # empty build side / empty probe side
    cases.append((np.zeros((0, 2), np.uint32), [0, 1], rng.integers(0, 4, size=(50, 2)), [1, 2], None))
    cases.append((rng.integers(0, 4, size=(50, 2)), [0, 1], np.zeros((0, 2), np.uint32), [1, 2], None))
    # large distinct keys (table growth, collisions)
    R = np.stack([np.arange(300000), rng.integers(0, 1 << 30, 300000)], axis=1)
    S = np.stack([rng.integers(0, 600000, 200000), rng.integers(0, 1 << 30, 200000)], axis=1)
    cases.append((R, [0, 1], S, [0, 2], None))
    for R, rv, S, sv, lab in cases:
        want, wv = hash_join(R, rv, S, sv, lab)
        got, gv = api.hash_join(engine, R, rv, S, sv, lab)
        assert gv == wv
        assert sorted(map(tuple, got.tolist())) == sorted(want)
        assert api.hash_join(engine, R, rv, S, sv, lab, count_only=True) == len(want)


@pytest.mark.gpu
@pytest.mark.parametrize("max_unit", [4, 6])
def test_join_counts_hprd(engine, max_unit):
    """HPRD-15 queries through the join path equal the reference's Q-mode
    counts and its recorded (C-mode) counts."""
    g, qs, counts = gd.hprd()
    ref = join_ref()["hprd"]
    dg = api.DataGraph.from_graph(g)
    for q, c, rc in zip(qs, counts, ref):
        r = api.match_join(engine, dg, q, "CFL_CFL_EXPLORE", max_unit_vertices=max_unit)
        assert len(r.units) >= 2
        assert r.count == c
        if rc is not None:
            assert r.count == rc


@pytest.mark.gpu
def test_join_counts_against_reference_q_mode(engine):
    """Larger seeded queries (16-24 vertices) on the scale-12 R-MAT graph:
    counts equal the reference's decomposition + join path and the plain
    path."""
    ref = join_ref()["rmat12"]
    g = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    dg = api.DataGraph.from_graph(g)
    checked = 0
    with api.Engine(arena_bytes=16 << 30) as big:
        for e in ref["queries"]:
            if e["count"] is None:
                continue  # the reference did not finish it within its time limit
            q = gd.query_from_rec(e["query"])
            r = api.match_join(big, dg, q, "CFL_CFL_EXPLORE", max_unit_vertices=12, time_limit=120)
            plain = api.match(big, dg, q, "CFL_CFL_EXPLORE", time_limit=120)
            assert r.count == plain.count == e["count"]
            checked += 1
    assert checked >= 4


@pytest.mark.gpu
def test_join_single_unit_and_empty(engine):
    """A query that fits one unit is counted without a join; a query with an
    unmatched label yields zero."""
    g, qs, counts = gd.hprd()
    dg = api.DataGraph.from_graph(g)
    r = api.match_join(engine, dg, qs[0], "GQL_GQL_GQL", max_unit_vertices=12)
    assert len(r.units) == 1 and r.count == counts[0]
    q = qs[1]
    lab = np.array(q.labels, np.uint32)
    lab[0] = 10_000  # a label no data vertex carries
    q2 = type(q).from_edges(q.num_vertices, lab, q.edge_list())
    r = api.match_join(engine, dg, q2, "CFL_CFL_EXPLORE", max_unit_vertices=4)
    assert r.count == 0


PATTERNS = ["STAR", "TWINTWIG", "SEED", "SKETCHTREE"]


@pytest.mark.gpu
@pytest.mark.parametrize("pattern", PATTERNS + ["COST"])
def test_join_patterns_match_reference_counts(pattern):
    """Every decomposition pattern (the reference's -Qpattern values with its
    own counts per pattern, and COST) and both join paradigms give the
    reference's Q-mode counts: HPRD-15 and the scale-12 R-MAT queries the
    reference's join path finished."""
    ref = join_ref()
    counts = ref["patterns"]["STAR" if pattern == "COST" else pattern]
    g, hq, _ = gd.hprd()
    hdg = api.DataGraph.from_graph(g)
    rg = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    rdg = api.DataGraph.from_graph(rg)
    cases = [(hdg, q, c, 4) for q, c in zip(hq, counts["hprd"])]
    cases += [(rdg, gd.query_from_rec(e["query"]), c, 12)
              for e, c in zip(ref["rmat12"]["queries"], counts["rmat12"])]
    checked = 0
    eng = api.Engine(arena_bytes=24 << 30)
    for dg, q, c, mu in cases:
        if c is None:
            continue
        for jm in ("LEFTDEEP", "BUSHY"):
            try:
                r = api.match_join(eng, dg, q, "CFL_CFL_EXPLORE", max_unit_vertices=mu, pattern=pattern,
                                   join_method=jm)
            except PsmError as e:
                # the reference's patterns have no unit bound: twin-twig covers
                # of large queries need more than 32 units, and small units
                # of large queries materialise relations beyond the arena
                assert pattern != "COST" and ("units" in str(e) or "arena" in str(e)), e
                continue
            assert r.count == c, (pattern, jm, q.num_vertices)
            checked += 1
    eng.close()
    hdg.close()
    rdg.close()
    assert checked >= 20
