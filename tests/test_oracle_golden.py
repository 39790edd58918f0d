"""The oracle restatement against what the reference itself computes.

Pins: the reference's recorded HPRD-15 counts (test_anony/C_output logs) and
candidate sets / tables / orders / counts dumped from the reference's own
compiled code on HPRD and on seeded synthetic workloads.
"""
import numpy as np
import pytest

from oracle.oracle import OracleGraph
from tests import golden_data as gd


@pytest.fixture(scope="module")
def hprd_oracle():
    g, qs, counts = gd.hprd()
    return OracleGraph(g), g, qs, counts


def _check_dump(r, d):
    assert len(r.candidates) == len(d["cands"])
    for u, (a, b) in enumerate(zip(r.candidates, d["cands"])):
        assert np.array_equal(a, np.array(b, np.uint32)), f"candidates of u{u}"
    for k, (off, adj) in gd.tables_of(d).items():
        assert np.array_equal(r.tables[k][0], off), f"table {k} offsets"
        assert np.array_equal(r.tables[k][1], adj), f"table {k} entries"
    assert r.memory_bytes == d["memory"]
    assert list(r.order) == d["order"]
    assert list(r.pivot[1:]) == d["pivot"][1:]


def test_hprd_graph_hash():
    g, _, _ = gd.hprd()
    assert gd.graph_sha(g) == gd.golden()["hprd"]["sha256"]


@pytest.mark.parametrize("qi", range(1, 11))
@pytest.mark.parametrize("method", ["GQL_GQL", "CFL_CFL", "NLF_GQL"])
def test_hprd_against_reference(hprd_oracle, qi, method):
    og, g, qs, counts = hprd_oracle
    filt, order = method.split("_")
    r = og.run(qs[qi - 1], filt, order)
    assert r.count == counts[qi - 1]
    _check_dump(r, gd.golden()["hprd"]["dumps"][f"{qi}:{method}"])


@pytest.mark.parametrize("name", [n for n, _ in gd.synthetic_cases()])
def test_synthetic_against_reference(name):
    case = dict(gd.synthetic_cases())[name]
    og = OracleGraph(gd.synthetic_graph(name))
    for j, entry in enumerate(case["queries"]):
        q = gd.query_from_rec(entry["query"])
        for m, d in entry["methods"].items():
            filt, order, _ = m.split("_")
            r = og.run(q, filt, order, cap=entry["cap"])
            assert r.count == d["count"], (name, j, m)
            _check_dump(r, d)


def test_embeddings_match_brute_force():
    """Full embedding sets of small queries against networkx's VF2."""
    nx = pytest.importorskip("networkx")
    from networkx.algorithms import isomorphism as iso
    g = gd.synthetic_graph("rmat12")
    og = OracleGraph(g)
    case = dict(gd.synthetic_cases())["rmat12"]
    G = nx.Graph()
    G.add_nodes_from((v, {"l": int(l)}) for v, l in enumerate(g.labels))
    G.add_edges_from(map(tuple, g.edge_list()))
    checked = 0
    for entry in case["queries"]:
        q = gd.query_from_rec(entry["query"])
        if q.num_vertices > 6:
            continue
        r = og.run(q, "CFL", "CFL", emit_limit=10**6)
        if r.count > 20000:
            continue
        Q = nx.Graph()
        Q.add_nodes_from((v, {"l": int(l)}) for v, l in enumerate(q.labels))
        Q.add_edges_from(map(tuple, q.edge_list()))
        gm = iso.GraphMatcher(G, Q, node_match=lambda a, b: a["l"] == b["l"])
        ref = set()
        for m in gm.subgraph_monomorphisms_iter():
            inv = {qv: dv for dv, qv in m.items()}
            ref.add(tuple(inv[i] for i in range(q.num_vertices)))
        got = set(map(tuple, r.embeddings.tolist()))
        assert got == ref
        checked += 1
    assert checked >= 3
