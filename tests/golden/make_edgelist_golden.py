"""Records the reference's edge-list converter output as golden fixtures.

Run in the development container, where the reference sources are mounted:

    python tests/golden/make_edgelist_golden.py [--ref /root/reference]

It builds oracle/_ref/EdgeListConverter.out from the reference's
matching/EdgeListToCSR.cpp (make -C oracle edgelist), runs it on a few edge
lists (comments, reversed and duplicate pairs, isolated ids, an unterminated
last line, a seeded random list, a self loop) and keeps its degree and
adjacency files. Its labels come from std::random_device, so only their
count is recorded.

Output: tests/golden/edgelist_ref.json.
"""
from __future__ import annotations

import argparse
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
BIN = ROOT / "oracle" / "_ref" / "EdgeListConverter.out"


def cases():
    yield "basic", "# a comment\n3 1\n0 2\n1 3\n2 8\n# another\n4 0\n8 1\n6 9", 5
    rng = np.random.default_rng(0x45444745)
    pairs = rng.integers(0, 500, size=(2000, 2))
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    pairs = np.concatenate([pairs, pairs[:40]])  # duplicates, in both orientations
    pairs[::3] = pairs[::3, ::-1]
    text = "# seeded random edge list\n" + "".join(f"{a} {b}\n" for a, b in pairs)
    yield "random", text, 32
    yield "selfloop", "0 1\n1 2\n2 2\n3 1\n", 4


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "edgelist", f"REF={args.ref}"], check=True)
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name, text, labels in cases():
            src = Path(td) / f"{name}.txt"
            src.write_text(text)
            pre = Path(td) / name
            subprocess.run([str(BIN), str(src), str(pre), str(labels)], check=True, capture_output=True)
            deg, adj, lab = (Path(f"{pre}_{s}.bin") for s in ("deg", "adj", "label"))
            rec = {"text": text, "num_labels": labels, "written": deg.exists()}
            if deg.exists():
                rec["deg"] = deg.read_bytes().hex()
                rec["adj"] = adj.read_bytes().hex()
                rec["label_bytes"] = lab.stat().st_size
            out[name] = rec
            print(name, rec["written"])
    (HERE / "edgelist_ref.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
