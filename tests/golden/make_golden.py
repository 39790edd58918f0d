"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Run in the development container, where the reference sources are mounted:

    python tests/golden/make_golden.py [--ref /root/reference]

Steps:
 1. builds the unmodified reference objects (oracle/Makefile, target `ref`)
    and links tests/golden/ref_dump.cpp against them;
 2. HPRD-15 (the reference's only dataset): stores the graph and its ten
    10-vertex queries in hprd15.npz, plus the #Embeddings the reference's
    recorded logs report (test_anony/C_output/HPRD/L15/Q10/*.txt);
 3. for HPRD and for seeded synthetic workloads (regenerated from their seeds
    by libpsm_gen at test time; a SHA-256 of the graph guards against drift)
    it records what the reference computes: candidate sets, candidate-edge
    tables, matching order and pivots (ref_dump), and the embedding count of
    the reference binary SubgraphMatching.out in "-QorCandi C" mode.

Output: hprd15.npz, golden_ref.json.gz (dumps + counts).
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from psm_benchmark_b200 import gen  # noqa: E402
from psm_benchmark_b200.graphs import Graph  # noqa: E402
from oracle.oracle import parse_ref_dump  # noqa: E402


def graph_sha(g: Graph) -> str:
    h = hashlib.sha256()
    for a in (g.off, g.nbr, g.labels):
        h.update(np.ascontiguousarray(a, np.uint32).tobytes())
    return h.hexdigest()


def build_ref(ref: Path) -> Path:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REF={ref}", "-j8"], check=True)
    objdir = ROOT / "oracle" / "_ref" / "obj"
    objs = [str(p) for p in objdir.rglob("*.o") if p.name != "StudyPerformance.o"]
    exe = ROOT / "oracle" / "_ref" / "ref_dump"
    subprocess.run(["/usr/bin/g++", "-std=c++20", "-O2", "-march=x86-64-v3", "-pthread", "-fopenmp", "-w",
                    f"-I{ref}", str(HERE / "ref_dump.cpp"), *objs, "-o", str(exe)], check=True)
    return exe


def run_ref_count(data_txt: str, query_txt: str, method: str, cap: int, tmp: Path) -> int:
    log = tmp / "log.txt"
    if log.exists():
        log.unlink()
    cmd = [str(ROOT / "oracle" / "_ref" / "SubgraphMatching.out"), "-d", data_txt, "-q", query_txt,
           "-threadnums", "1", "-num", str(cap) if cap else "MAX", "-time_limit", "600",
           "-OutputFile", str(log), "-QorCandi", "C", "-split", "linear", "-schedule", "busy2idlenostop",
           "-BackMethods", method]
    subprocess.run(cmd, check=True, capture_output=True)
    text = log.read_text()
    assert "Overtime: 0" in text, text[-400:]
    return int(re.findall(r"#Embeddings: (\d+)", text)[-1])


def dump(exe: Path, data_txt: str, query_txt: str, filt: str, order: str) -> dict:
    out = subprocess.run([str(exe), data_txt, query_txt, filt, order], check=True, capture_output=True,
                         text=True).stdout
    d = parse_ref_dump(out)
    return {"cands": [c.tolist() for c in d["cands"]],
            "tables": [[a, b, off.tolist(), adj.tolist()] for (a, b), (off, adj) in sorted(d["tables"].items())],
            "order": d["order"].tolist(), "pivot": d["pivot"].tolist(), "memory": d["memory"]}


def qrec(q: Graph) -> dict:
    return {"labels": q.labels.tolist(), "edges": q.edge_list().tolist()}


def write_query(q: Graph, path: Path) -> str:
    path.parent.mkdir(parents=True, exist_ok=True)
    q.write_text(path)
    return str(path)


def synthetic_cases():
    """(name, graph, queries, [(filter, order, engine)], cap)."""
    w1 = gen.plain_small(num_queries=40)
    yield ("plain_small", {"kind": "plain_small"}, w1.graph, w1.queries,
           [("GQL", "GQL", "GQL"), ("CFL", "CFL", "EXPLORE")], 0)
    # The R-MAT workload at a reduced scale so the single-threaded reference
    # finishes in seconds; same generator, labels and query extraction.
    g2 = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
    qs = gen.make_queries(g2, [4, 6, 8, 12] * 6, gen.BASE_SEED + 2)
    yield ("rmat12", {"kind": "rmat", "index": 2, "scale": 12, "edge_factor": 8, "num_labels": 32,
                      "sizes": [4, 6, 8, 12] * 6}, g2, qs,
           [("CFL", "CFL", "EXPLORE"), ("GQL", "GQL", "GQL")], 100000)


# Hand-made edge cases (stars of same-label leaves around hubs) can have
# billions of embeddings; they are counted under this cap.
EDGE_CASE_CAP = 1000000


def edge_queries(g: Graph):
    """Hand-made edge cases on a data graph: single edge, triangle, a label
    that no data vertex carries (empty candidate set), a star."""
    lab = g.labels
    l0, l1 = int(lab[0]), int(lab[g.neighbors(0)[0]]) if g.degree(0) else int(lab[0])
    out = [
        Graph.from_edges(2, [l0, l1], [(0, 1)]),
        Graph.from_edges(3, [l0, l0, l1], [(0, 1), (1, 2), (0, 2)]),
        Graph.from_edges(5, [l1, l0, l0, l0, l0], [(0, 1), (0, 2), (0, 3), (0, 4)]),
    ]
    # A label below the data graph's largest label that no vertex carries
    # (labels beyond the largest one index past the reference's label index).
    present = np.zeros(int(lab.max()) + 1, dtype=bool)
    present[lab] = True
    missing = np.flatnonzero(~present)
    if missing.size:
        out.append(Graph.from_edges(3, [l0, int(missing[0]), l1], [(0, 1), (1, 2)]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    ref = Path(args.ref)
    exe = build_ref(ref)
    out = {"hprd": {}, "synthetic": []}
    with tempfile.TemporaryDirectory() as td:
        tmp = Path(td)
        # --- HPRD ---------------------------------------------------------
        hdir = ref / "datasets" / "HPRD" / "L15"
        G = Graph.read_text(hdir / "HPRD-15.txt")
        qs = [Graph.read_text(hdir / "Q10" / f"Q10-{i}.txt") for i in range(1, 11)]
        rec = {}
        for i in range(1, 11):
            text = (ref / "test_anony" / "C_output" / "HPRD" / "L15" / "Q10" / f"Q10-{i}.txt").read_text()
            counts = set(int(x) for x in re.findall(r"#Embeddings: (\d+)", text))
            assert len(counts) == 1, counts
            rec[i] = counts.pop()
        np.savez_compressed(HERE / "hprd15.npz", off=G.off, nbr=G.nbr, labels=G.labels,
                            q_labels=np.array([q.labels for q in qs], dtype=np.uint32),
                            q_edges=np.array([np.pad(q.edge_list(), ((0, 20 - q.num_edges), (0, 0)),
                                                     constant_values=-1) for q in qs], dtype=np.int64),
                            recorded_counts=np.array([rec[i] for i in range(1, 11)], dtype=np.uint64))
        out["hprd"] = {"sha256": graph_sha(G), "recorded_counts": [rec[i] for i in range(1, 11)], "dumps": {}}
        for i in range(1, 11):
            qp = str(hdir / "Q10" / f"Q10-{i}.txt")
            for filt, order in [("GQL", "GQL"), ("CFL", "CFL"), ("NLF", "GQL")]:
                out["hprd"]["dumps"][f"{i}:{filt}_{order}"] = dump(exe, str(hdir / "HPRD-15.txt"), qp, filt, order)
        # --- synthetic ----------------------------------------------------
        for name, spec, g, queries, methods, cap in synthetic_cases():
            dpath = tmp / "d1" / "d2" / f"{name}.txt"
            dpath.parent.mkdir(parents=True, exist_ok=True)
            g.write_text(dpath)
            case = {"name": name, "spec": spec, "sha256": graph_sha(g), "cap": cap, "queries": []}
            all_q = list(queries) + edge_queries(g)
            for j, q in enumerate(all_q):
                qpath = write_query(q, tmp / "q1" / "q2" / "q3" / f"{name}_{j}.txt")
                edge_case = j >= len(queries)
                qcap = EDGE_CASE_CAP if edge_case else cap
                entry = {"query": qrec(q), "edge_case": edge_case, "cap": qcap, "methods": {}}
                for filt, order, engine in methods:
                    m = f"{filt}_{order}_{engine}"
                    d = dump(exe, str(dpath), qpath, filt, order)
                    d["count"] = run_ref_count(str(dpath), qpath, m, qcap, tmp)
                    entry["methods"][m] = d
                case["queries"].append(entry)
                print(name, j, {m: v["count"] for m, v in entry["methods"].items()}, flush=True)
            out["synthetic"].append(case)
    with gzip.open(HERE / "golden_ref.json.gz", "wt") as f:
        json.dump(out, f)
    print("wrote", HERE / "golden_ref.json.gz", os.path.getsize(HERE / "golden_ref.json.gz"), "bytes")


if __name__ == "__main__":
    main()
