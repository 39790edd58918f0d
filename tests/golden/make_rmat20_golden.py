"""Pins the device path to the reference on the plain benchmark's own graph.

The plain benchmark workload (R-MAT scale 20, edge factor 8, 32 uniform
labels, 12- and 16-vertex random-walk queries, cap 1e9) has more than 1e9
embeddings in every query: in probes of about 100 further 12- and 16-vertex
random-walk queries of this graph (sparse, dense, extracted around hubs or
from a degree-3 start) none finished below the cap within the reference's
time limit, each counting 1e7-5e7 embeddings per second. Exact counts on
this graph are therefore pinned where the reference finishes, and the rest of
the path is pinned stage by stage:

 1. for the first 24 queries of each size of the benchmark workload itself:
    SHA-256 digests of the reference's candidate sets, candidate-edge tables,
    matching order and memory cost (tests/golden/ref_dump.cpp) under
    CFL/CFL and GQL/GQL;
 2. for the 4- and 6-vertex queries of the batched workload on the same
    graph (2,000 random-walk queries of 4-32 vertices): the counts of the
    unmodified SubgraphMatching.out (oracle/Makefile, -threadnums 1, cap
    1e9) under CFL_CFL_EXPLORE and GQL_GQL_GQL where both finish with
    Overtime: 0, and the same digests.

Run in the development container, where the reference sources are mounted:

    python tests/golden/make_rmat20_golden.py [--ref /root/reference] [--jobs 7]

Output: tests/golden/rmat20_ref.json (queries, counts, digests; the graph is
regenerated from its seed at test time and checked by SHA-256).
"""
from __future__ import annotations

import argparse
import json
import re
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from psm_benchmark_b200 import gen  # noqa: E402
from oracle.oracle import parse_ref_dump  # noqa: E402
from tests.golden.make_golden import build_ref, qrec  # noqa: E402
from tests.golden_data import digest_cands, digest_tables, graph_sha  # noqa: E402

CAP = 10**9
METHODS = ("CFL_CFL_EXPLORE", "GQL_GQL_GQL")


def run_ref(data_txt: str, query_txt: str, method: str, limit: int, log: Path):
    if log.exists():
        log.unlink()
    cmd = [str(ROOT / "oracle" / "_ref" / "SubgraphMatching.out"), "-d", data_txt, "-q", query_txt,
           "-threadnums", "1", "-num", str(CAP), "-time_limit", str(limit), "-OutputFile", str(log),
           "-QorCandi", "C", "-split", "linear", "-schedule", "busy2idlenostop", "-BackMethods", method]
    subprocess.run(cmd, check=True, capture_output=True, timeout=limit + 300)
    text = log.read_text()
    count = int(re.findall(r"#Embeddings: (\d+)", text)[-1])
    over = int(re.findall(r"Overtime: (\d+)", text)[-1])
    total = float(re.findall(r"Total time \(seconds\): ([0-9.e+-]+)", text)[-1])
    return count, over, total


def digests(exe: Path, data_txt: str, query_txt: str, filt: str, order: str) -> dict:
    out = subprocess.run([str(exe), data_txt, query_txt, filt, order], check=True, capture_output=True,
                         text=True).stdout
    d = parse_ref_dump(out)
    return {"cands_sha": digest_cands(d["cands"]),
            "cand_counts": [int(len(c)) for c in d["cands"]],
            "tables_sha": digest_tables(d["tables"]),
            "order": d["order"].tolist(), "pivot": d["pivot"].tolist(), "memory": d["memory"]}


def pin(exe, data_txt, tmp, name, queries, limit, jobs, counts=True):
    """Reference digests (and counts) of `queries` [(workload index, query)];
    with counts, keeps the queries both methods finish."""
    qdir = tmp / "q1" / "q2" / "q3"
    qdir.mkdir(parents=True, exist_ok=True)

    def one(item):
        idx, q = item
        qp = qdir / f"{name}_{idx}.txt"
        q.write_text(qp)
        entry = {"index": idx, "query": qrec(q), "size": q.num_vertices, "methods": {}}
        for m in METHODS:
            f, o, _ = m.split("_")
            d = digests(exe, data_txt, str(qp), f, o)
            if counts:
                c, over, tot = run_ref(data_txt, str(qp), m, limit, tmp / f"log_{name}_{idx}.txt")
                if over or c >= CAP:
                    return None
                d.update(count=c, ref_total_s=tot)
            entry["methods"][m] = d
        print(name, idx, q.num_vertices, {m: v.get("count") for m, v in entry["methods"].items()}, flush=True)
        return entry

    with ThreadPoolExecutor(jobs) as pool:
        return [e for e in pool.map(one, queries) if e is not None]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--jobs", type=int, default=7)
    ap.add_argument("--bench-per-size", type=int, default=24)
    ap.add_argument("--small", type=int, default=40, help="batched-workload queries tried per small size")
    ap.add_argument("--limit", type=int, default=120, help="reference time limit per run (s)")
    args = ap.parse_args()
    exe = build_ref(Path(args.ref))
    bench = gen.plain_rmat()
    g = bench.graph
    mixed = gen.batched(graph=g)
    out = {"cap": CAP, "spec": {"index": 2, "scale": 20, "edge_factor": 8, "num_labels": 32},
           "sha256": graph_sha(g), "bench": [], "small": []}
    with tempfile.TemporaryDirectory() as td:
        tmp = Path(td)
        dpath = tmp / "d1" / "d2" / "rmat20.txt"
        dpath.parent.mkdir(parents=True, exist_ok=True)
        gen.write_text(g, dpath)
        for k in (12, 16):
            items = [(i, q) for i, q in enumerate(bench.queries) if q.num_vertices == k][: args.bench_per_size]
            out["bench"] += pin(exe, str(dpath), tmp, f"bench{k}", items, args.limit, args.jobs, counts=False)
        for k in (4, 6):
            items = [(i, q) for i, q in enumerate(mixed.queries) if q.num_vertices == k][: args.small]
            kept = pin(exe, str(dpath), tmp, f"mixed{k}", items, args.limit, args.jobs)
            print(f"size {k}: kept {len(kept)} of {len(items)}", flush=True)
            out["small"] += kept
    (HERE / "rmat20_ref.json").write_text(json.dumps(out))
    print("wrote", HERE / "rmat20_ref.json")


if __name__ == "__main__":
    main()
