"""Shared fixtures for the GPU tests."""
import numpy as np
import pytest

from psm_benchmark_b200 import api


@pytest.fixture(scope="session")
def engine():
    e = api.Engine(arena_bytes=2 << 30)
    yield e
    e.close()


def check_run_against_dump(run, d, check_order=True):
    """Candidates, tables, order and memory cost of a Run against a dump of
    the reference (or the oracle), in original data ids."""
    n = run.query.num_vertices
    for u in range(n):
        assert np.array_equal(run.candidates(u), np.asarray(d["cands"][u], np.uint32)), f"candidates u{u}"
    if any(len(c) == 0 for c in d["cands"]):
        return
    for a, b, off, adj in d["tables"]:
        o, e = run.table(a, b)
        assert np.array_equal(o, np.asarray(off, np.uint32)), f"T[{a}][{b}] offsets"
        assert np.array_equal(e, np.asarray(adj, np.uint32)), f"T[{a}][{b}] entries"
    assert run.result.memory_bytes == d["memory"]
    if check_order:
        o, p = run.order()
        assert list(o) == list(d["order"]), (list(o), d["order"])
        assert list(p[1:]) == list(d["pivot"][1:])
