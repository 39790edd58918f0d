"""Records the reference's decomposition + join ("-QorCandi Q") counts as
golden fixtures for the join path.

Run in the development container, where the reference sources are mounted
and oracle/_ref/SubgraphMatching.out has been built (make -C oracle ref):

    python tests/golden/make_join_golden.py [--ref /root/reference]

For the HPRD-15 queries and for seeded larger queries (16-24 vertices) on the
scale-12 R-MAT graph of the synthetic fixtures, it runs the unmodified
reference binary with -QorCandi Q -Qpattern P -JoinMethod LEFTDEEP
-threadnums 1 (the reference's join path; it aborts with more threads) for
each decomposition pattern P in STAR, TWINTWIG, SEED and SKETCHTREE, and
keeps the runs that finished within the time limit (Overtime: 0). The
top-level "hprd" / "rmat12" counts are the STAR runs; "patterns" holds every
pattern's.

Output: tests/golden/join_ref.json (queries as label/edge lists + counts).
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
from psm_benchmark_b200.graphs import Graph  # noqa: E402

REF_BIN = ROOT / "oracle" / "_ref" / "SubgraphMatching.out"
TIME_LIMIT = 60
METHOD = "CFL_CFL_EXPLORE"


def run_q(data: Path, query: Path, log: Path, pattern: str = "STAR"):
    if log.exists():
        log.unlink()
    cmd = [str(REF_BIN), "-d", str(data), "-q", str(query), "-num", "MAX", "-time_limit", str(TIME_LIMIT),
           "-OutputFile", str(log), "-QorCandi", "Q", "-Qpattern", pattern, "-JoinMethod", "LEFTDEEP",
           "-threadnums", "1", "-BackMethods", METHOD]
    try:
        subprocess.run(cmd, check=True, capture_output=True, timeout=TIME_LIMIT + 60)
    except (subprocess.CalledProcessError, subprocess.TimeoutExpired):
        return None
    text = log.read_text()
    over = int(re.findall(r"Overtime: (\d+)", text)[-1])
    if over:
        return None
    return int(re.findall(r"#Embeddings: (\d+)", text)[-1])


def qrec(q: Graph):
    return {"labels": [int(x) for x in q.labels], "edges": [[int(a), int(b)] for a, b in q.edge_list()]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    ref = Path(args.ref)
    if not REF_BIN.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REF={ref}", "-j8"], check=True)
    out = {"method": METHOD, "pattern": "STAR", "join": "LEFTDEEP", "hprd": [], "rmat12": {}, "patterns": {}}
    patterns = ("STAR", "TWINTWIG", "SEED", "SKETCHTREE")
    with tempfile.TemporaryDirectory() as td:
        # the reference needs >= 3 / 4 slashes in the data / query paths
        base = Path(td) / "a" / "b" / "c"
        (base / "q").mkdir(parents=True)
        hdir = ref / "datasets" / "HPRD" / "L15"
        g = gen.make_graph("rmat", 2, scale=12, edge_factor=8, num_labels=32)
        data = base / "rmat12.txt"
        gen.write_text(g, data)
        sizes = [16, 16, 20, 20, 24, 24] * 2
        seed = gen.BASE_SEED + 4
        qs = gen.make_queries(g, sizes, seed)
        for j, q in enumerate(qs):
            q.write_text(base / "q" / f"q{j}.txt")
        jobs = [(p, "hprd", i, hdir / "HPRD-15.txt", hdir / "Q10" / f"Q10-{i + 1}.txt") for p in patterns
                for i in range(10)]
        jobs += [(p, "rmat12", j, data, base / "q" / f"q{j}.txt") for p in patterns for j in range(len(qs))]

        def one(job):
            p, name, i, d, qp = job
            c = run_q(d, qp, Path(td) / f"out_{p}_{name}_{i}.log", p)
            print(p, name, i, c, flush=True)
            return job, c

        with ThreadPoolExecutor(7) as pool:
            results = list(pool.map(one, jobs))
        for p in patterns:
            out["patterns"][p] = {"hprd": [None] * 10, "rmat12": [None] * len(qs)}
        for (p, name, i, _, _), c in results:
            out["patterns"][p][name][i] = c
        out["hprd"] = out["patterns"]["STAR"]["hprd"]
        out["rmat12"] = {"sizes": sizes, "seed": seed,
                         "queries": [{"query": qrec(q), "count": out["patterns"]["STAR"]["rmat12"][j]}
                                     for j, q in enumerate(qs)]}
    (HERE / "join_ref.json").write_text(json.dumps(out))


if __name__ == "__main__":
    main()
