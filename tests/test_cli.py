"""psm_match, the drop-in for the reference's SubgraphMatching.out command
line: flag handling and the log block (matching/Args.cpp:517-535 prefixed by
utility/statistics/Logs.h:88-96).

The CPU tests check flag and error handling; the GPU test runs the HPRD-15
queries the way the reference's own experiment script does
(-QorCandi C -BackMethods ...) and reads '#Embeddings:' back from the log.
"""
import re
import subprocess

import pytest

from psm_benchmark_b200 import build
from tests.golden_data import hprd


@pytest.fixture(scope="module")
def cli():
    build.build_core()
    return build.build_cli()


def run(cli, args):
    return subprocess.run([str(cli), *args], capture_output=True, text=True, timeout=300)


def test_undefined_split_mode_is_rejected(cli, tmp_path):
    log = tmp_path / "out.log"
    p = run(cli, ["-d", "x", "-q", "y", "-QorCandi", "NOSPLIT", "-OutputFile", str(log)])
    assert p.returncode == 1
    assert log.read_text() == "[Thread 1] Error: The split mode is not defined.\n"


def test_undefined_query_pattern_is_rejected(cli, tmp_path):
    log = tmp_path / "out.log"
    p = run(cli, ["-d", "x", "-q", "y", "-QorCandi", "Q", "-Qpattern", "CHAIN", "-OutputFile", str(log)])
    assert p.returncode == 1
    assert log.read_text() == "[Thread 1] Error: The split pattern 'CHAIN' is not defined.\n"
    p = run(cli, ["-d", "x", "-q", "y", "-QorCandi", "Q", "-JoinMethod", "RIGHTDEEP", "-OutputFile", str(log)])
    assert p.returncode == 1


def test_missing_graph_files(cli, tmp_path):
    p = run(cli, ["-d", str(tmp_path / "missing.txt"), "-q", str(tmp_path / "q.txt"), "-QorCandi", "C"])
    assert p.returncode == 1
    assert "psm_match:" in p.stderr


def parse_blocks(text):
    blocks, cur = [], None
    for line in text.splitlines():
        assert line.startswith("[Thread 1] ")
        body = line[len("[Thread 1] "):]
        if body == "Start the query":
            cur = {}
        elif body == "End the query":
            blocks.append(cur)
            cur = None
        elif cur is not None and ": " in body:
            k, v = body.split(": ", 1)
            cur[k] = v
    return blocks


@pytest.mark.gpu
def test_hprd_counts_through_cli(cli, tmp_path):
    g, qs, counts = hprd()
    data = tmp_path / "datasets" / "HPRD" / "L15" / "HPRD-15.txt"
    data.parent.mkdir(parents=True)
    g.write_text(data)
    for i, (q, want) in enumerate(zip(qs, counts)):
        qf = tmp_path / "datasets" / "HPRD" / "L15" / "Q10" / f"Q10-{i + 1}.txt"
        qf.parent.mkdir(exist_ok=True)
        q.write_text(qf)
        log = tmp_path / f"out{i}.log"
        p = run(cli, ["-d", str(data), "-q", str(qf), "-num", "MAX", "-time_limit", "60", "-OutputFile", str(log),
                      "-QorCandi", "C", "-threadnums", "1,4", "-split", "linear", "-schedule", "busy2idlenostop",
                      "-BackMethods", "GQL_GQL_GQL,CFL_CFL_EXPLORE,NLF_GQL_LFTJ,CFL_CFL_DPiso"])
        assert p.returncode == 0, p.stderr
        blocks = parse_blocks(log.read_text())
        assert len(blocks) == 8
        for b in blocks:
            assert b["Input Data Graph File"] == "HPRD/L15/HPRD-15.txt"
            assert int(b["#Embeddings"]) == want
            assert b["Overtime"] == "0"
            assert re.fullmatch(r"[0-9.e+-]+", b["Total time (seconds)"])
        assert [b["Num Threads"] for b in blocks] == ["1"] * 4 + ["4"] * 4
        assert [b["Engine Type"] for b in blocks[:4]] == ["GQL", "EXPLORE", "LFTJ", "DPiso"]


@pytest.mark.gpu
def test_unsupported_filter_is_reported(cli, tmp_path):
    g, qs, counts = hprd()
    data = tmp_path / "d.txt"
    g.write_text(data)
    qf = tmp_path / "q.txt"
    qs[0].write_text(qf)
    log = tmp_path / "out.log"
    p = run(cli, ["-d", str(data), "-q", str(qf), "-QorCandi", "C", "-OutputFile", str(log),
                  "-BackMethods", "DPiso_DPiso_LFTJ,CFL_CFL_LFTJ"])
    assert p.returncode == 1
    text = log.read_text()
    assert "The specified filter type 'DPiso' is not supported." in text
    blocks = parse_blocks(text)
    assert len(blocks) == 1 and int(blocks[0]["#Embeddings"]) == counts[0]


@pytest.mark.gpu
def test_hprd_counts_through_cli_q_mode(cli, tmp_path):
    """-QorCandi Q (decomposition + join) gives the same #Embeddings."""
    g, qs, counts = hprd()
    data = tmp_path / "d.txt"
    g.write_text(data)
    for i in (0, 3, 6):
        qf = tmp_path / f"q{i}.txt"
        qs[i].write_text(qf)
        log = tmp_path / f"q{i}.log"
        p = run(cli, ["-d", str(data), "-q", str(qf), "-QorCandi", "Q", "-Qpattern", "STAR", "-JoinMethod", "LEFTDEEP",
                      "-threadnums", "1", "-OutputFile", str(log), "-BackMethods", "CFL_CFL_EXPLORE", "-max_unit", "4"])
        assert p.returncode == 0, p.stderr
        text = log.read_text()
        blocks = parse_blocks(text)
        assert len(blocks) == 1
        assert int(blocks[0]["#Embeddings"]) == counts[i]
        assert blocks[0]["QuerySplit Pattern"] == "STAR"
        assert int(re.search(r"subgraph count == (\d+)", text).group(1)) >= 2


@pytest.mark.gpu
@pytest.mark.parametrize("pattern,join", [("SKETCHTREE", "LEFTDEEP"), ("TWINTWIG", "BUSHY"), ("COST", "BUSHY")])
def test_q_mode_patterns_through_cli(cli, tmp_path, pattern, join):
    """-Qpattern / -JoinMethod choose the decomposition and join tree; the
    count is the reference's for every choice."""
    g, qs, counts = hprd()
    data = tmp_path / "d.txt"
    g.write_text(data)
    for i in (1, 4):
        qf = tmp_path / f"q{i}.txt"
        qs[i].write_text(qf)
        log = tmp_path / f"q{i}_{pattern}.log"
        p = run(cli, ["-d", str(data), "-q", str(qf), "-QorCandi", "Q", "-Qpattern", pattern, "-JoinMethod", join,
                      "-threadnums", "1", "-OutputFile", str(log), "-BackMethods", "CFL_CFL_EXPLORE", "-max_unit", "4"])
        assert p.returncode == 0, p.stderr
        blocks = parse_blocks(log.read_text())
        assert int(blocks[0]["#Embeddings"]) == counts[i]
        assert blocks[0]["QuerySplit Pattern"] == pattern
        assert blocks[0]["Join Paradigm"] == join
