"""Loads the committed golden fixtures (see tests/golden/make_golden.py).

Synthetic data graphs are regenerated from their seeds by libpsm_gen and
checked against the SHA-256 recorded when the fixtures were made.
"""
from __future__ import annotations

import gzip
import hashlib
import json
from functools import lru_cache
from pathlib import Path

import numpy as np

from psm_benchmark_b200 import gen
from psm_benchmark_b200.graphs import Graph

GOLDEN = Path(__file__).resolve().parent / "golden"


def graph_sha(g: Graph) -> str:
    h = hashlib.sha256()
    for a in (g.off, g.nbr, g.labels):
        h.update(np.ascontiguousarray(a, np.uint32).tobytes())
    return h.hexdigest()


@lru_cache(maxsize=1)
def golden():
    with gzip.open(GOLDEN / "golden_ref.json.gz", "rt") as f:
        return json.load(f)


@lru_cache(maxsize=1)
def hprd():
    """(graph, [10 queries], recorded counts) of the reference's HPRD-15 set."""
    z = np.load(GOLDEN / "hprd15.npz")
    g = Graph(off=z["off"], nbr=z["nbr"], labels=z["labels"])
    qs = []
    for lab, e in zip(z["q_labels"], z["q_edges"]):
        e = e[e[:, 0] >= 0]
        qs.append(Graph.from_edges(len(lab), lab, e))
    return g, qs, [int(x) for x in z["recorded_counts"]]


def query_from_rec(rec) -> Graph:
    return Graph.from_edges(len(rec["labels"]), rec["labels"], rec["edges"])


@lru_cache(maxsize=4)
def synthetic_graph(name: str) -> Graph:
    case = next(c for c in golden()["synthetic"] if c["name"] == name)
    spec = case["spec"]
    if spec["kind"] == "plain_small":
        g = gen.make_graph("chung_lu", 1, n=9460, num_labels=307, zipf_s=1.1)
    else:
        g = gen.make_graph("rmat", spec["index"], scale=spec["scale"], edge_factor=spec["edge_factor"],
                           num_labels=spec["num_labels"])
    if graph_sha(g) != case["sha256"]:
        raise AssertionError(f"generator drift: {name} graph hash changed")
    return g


def synthetic_cases():
    for case in golden()["synthetic"]:
        yield case["name"], case


def tables_of(d):
    return {(a, b): (np.array(off, np.uint32), np.array(adj, np.uint32)) for a, b, off, adj in d["tables"]}


def digest_cands(cands) -> str:
    """SHA-256 of candidate sets (a list, by query vertex, of sorted data ids)."""
    h = hashlib.sha256()
    for c in cands:
        c = np.ascontiguousarray(c, np.uint32)
        h.update(np.uint32(len(c)).tobytes())
        h.update(c.tobytes())
    return h.hexdigest()


def digest_tables(tables) -> str:
    """SHA-256 of candidate-edge tables {(a, b): (offsets, entries)}, in (a, b) order."""
    h = hashlib.sha256()
    for (a, b) in sorted(tables):
        off, adj = (np.ascontiguousarray(x, np.uint32) for x in tables[(a, b)])
        h.update(np.array([a, b, len(off), len(adj)], np.uint32).tobytes())
        h.update(off.tobytes())
        h.update(adj.tobytes())
    return h.hexdigest()


@lru_cache(maxsize=1)
def rmat20():
    """Pinned queries on the plain benchmark's graph (make_rmat20_golden.py)."""
    p = GOLDEN / "rmat20_ref.json"
    return json.loads(p.read_text()) if p.exists() else None


def pinned_graph(rec) -> Graph:
    spec = rec["spec"]
    g = gen.make_graph("rmat", spec["index"], scale=spec["scale"], edge_factor=spec["edge_factor"],
                       num_labels=spec["num_labels"])
    if graph_sha(g) != rec["sha256"]:
        raise AssertionError(f"generator drift: {rec.get('name', 'rmat20')} graph hash changed")
    return g
