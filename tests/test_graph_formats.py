"""Graph file formats: the reference's text format and its binary format
(Graph::loadGraphFromFileCompressed / storeComparessedGraph,
graph/graph.cpp:221-403; GraphConverter). The CPU tests check the bytes
against the format's layout; the GPU test matches queries on a graph loaded
from the binary files."""
import numpy as np
import pytest

from psm_benchmark_b200 import api
from tests import golden_data as gd
from tests.gpu_common import engine  # noqa: F401


def expected_files(g):
    """The three files of the reference's binary format, restated with numpy."""
    off = np.asarray(g.off, np.int64)
    V = g.num_vertices
    head = np.array([4, V, off[-1] // 2], np.uint32)
    deg = np.diff(off).astype(np.uint32)
    return (np.concatenate([head, deg]).tobytes(), np.asarray(g.nbr, np.uint32).tobytes(),
            np.asarray(g.labels, np.uint32).tobytes())


def test_store_matches_the_reference_layout(tmp_path):
    g, _, _ = gd.hprd()
    api.store_binary(g, tmp_path / "hprd")
    want = expected_files(g)
    got = [(tmp_path / f"hprd_{s}.bin").read_bytes() for s in ("deg", "adj", "label")]
    assert got == list(want)


def test_convert_text_equals_store(tmp_path):
    g = gd.synthetic_graph("rmat12")
    g.write_text(tmp_path / "g.txt")
    api.convert_text(tmp_path / "g.txt", tmp_path / "conv")
    api.store_binary(g, tmp_path / "direct")
    for s in ("deg", "adj", "label"):
        assert (tmp_path / f"conv_{s}.bin").read_bytes() == (tmp_path / f"direct_{s}.bin").read_bytes()


def test_malformed_binary_is_rejected(tmp_path):
    g, _, _ = gd.hprd()
    api.store_binary(g, tmp_path / "h")
    raw = (tmp_path / "h_adj.bin").read_bytes()
    (tmp_path / "h_adj.bin").write_bytes(raw[: len(raw) // 2])  # truncated adjacency
    from psm_benchmark_b200.native import PsmError
    with pytest.raises(PsmError):
        api.DataGraph.load_binary(tmp_path / "h")


@pytest.mark.gpu
def test_binary_graph_matches_like_text(engine, tmp_path):
    g, qs, counts = gd.hprd()
    api.store_binary(g, tmp_path / "hprd")
    dg = api.DataGraph.load_binary(tmp_path / "hprd")
    for q, c in zip(qs, counts):
        assert api.match(engine, dg, q, "CFL_CFL_EXPLORE").count == c


EDGELIST_REF = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "edgelist_ref.json"


@pytest.mark.parametrize("name", ["basic", "random", "selfloop"])
def test_edgelist_matches_the_reference_converter(tmp_path, name):
    """Degree and adjacency files byte-identical to the reference's
    EdgeListConverter (matching/EdgeListToCSR.cpp) on the recorded inputs
    (tests/golden/make_edgelist_golden.py); a self loop writes nothing."""
    import json
    from psm_benchmark_b200.native import PsmError
    rec = json.loads(EDGELIST_REF.read_text())[name]
    src = tmp_path / "e.txt"
    src.write_text(rec["text"])
    pre = tmp_path / "g"
    if not rec["written"]:
        with pytest.raises(PsmError, match="self loop"):
            api.convert_edgelist(src, pre, rec["num_labels"])
        assert not list(tmp_path.glob("g_*"))
        return
    api.convert_edgelist(src, pre, rec["num_labels"], seed=3)
    assert (tmp_path / "g_deg.bin").read_bytes() == bytes.fromhex(rec["deg"])
    assert (tmp_path / "g_adj.bin").read_bytes() == bytes.fromhex(rec["adj"])
    lab = np.fromfile(tmp_path / "g_label.bin", np.uint32)
    assert lab.nbytes == rec["label_bytes"]
    assert lab.max() < rec["num_labels"]


def test_edgelist_labels_follow_the_seed(tmp_path):
    src = tmp_path / "e.txt"
    src.write_text("".join(f"{i} {i + 1}\n" for i in range(300)))
    got = {}
    for seed in (1, 1, 2):
        api.convert_edgelist(src, tmp_path / f"s{seed}", 16, seed=seed)
        lab = np.fromfile(tmp_path / f"s{seed}_label.bin", np.uint32)
        assert lab.size == 301 and lab.max() < 16
        assert seed not in got or np.array_equal(got[seed], lab)
        got[seed] = lab
    assert not np.array_equal(got[1], got[2])
    assert len(np.unique(got[1])) > 8


@pytest.mark.parametrize("text,labels", [("0 1\n2\n", 4), ("0 -1\n", 4), ("0 x\n", 4), ("0 1\n", 0)])
def test_edgelist_rejects_malformed_input(tmp_path, text, labels):
    from psm_benchmark_b200.native import PsmError
    src = tmp_path / "e.txt"
    src.write_text(text)
    with pytest.raises(PsmError):
        api.convert_edgelist(src, tmp_path / "g", labels)
