"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes front end of liboracle.so, the CPU restatement of the reference's
subgraph-matching path (see psm_oracle.cpp). Imported only by tests/, the
smoke check and the bench's CPU-baseline leg, as the checker.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
FILTERS = {"NLF": 0, "GQL": 1, "CFL": 2}
ORDERS = {"GQL": 0, "CFL": 1}


def build() -> Path:
    lib = HERE / "liboracle.so"
    src = HERE / "psm_oracle.cpp"
    if not lib.exists() or lib.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    return lib


@lru_cache(maxsize=1)
def _lib():
    lib = C.CDLL(str(build()))
    u32p = C.POINTER(C.c_uint32)
    lib.orc_graph_new.argtypes = [u32p, u32p, u32p, C.c_uint32]
    lib.orc_graph_new.restype = C.c_void_p
    lib.orc_graph_free.argtypes = [C.c_void_p]
    lib.orc_run.argtypes = [C.c_void_p, u32p, u32p, u32p, C.c_uint32, C.c_int, C.c_int, C.c_uint64, C.c_uint64]
    lib.orc_run.restype = C.c_void_p
    for name, rt in [("orc_res_count", C.c_uint64), ("orc_res_calls", C.c_uint64), ("orc_res_memory", C.c_uint64),
                     ("orc_res_num_emb", C.c_uint64), ("orc_res_filter_ok", C.c_int)]:
        getattr(lib, name).argtypes = [C.c_void_p]
        getattr(lib, name).restype = rt
    lib.orc_res_cand_count.argtypes = [C.c_void_p, C.c_uint32]
    lib.orc_res_cand_count.restype = C.c_uint32
    lib.orc_res_cands.argtypes = [C.c_void_p, C.c_uint32, u32p]
    lib.orc_res_table_nnz.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
    lib.orc_res_table_nnz.restype = C.c_uint32
    lib.orc_res_table.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, u32p, u32p]
    lib.orc_res_order.argtypes = [C.c_void_p, u32p, u32p]
    lib.orc_res_emb.argtypes = [C.c_void_p, u32p]
    u64p = C.POINTER(C.c_uint64)
    lib.orc_res_depth_stats.argtypes = [C.c_void_p, u64p, u64p, u64p]
    lib.orc_res_free.argtypes = [C.c_void_p]
    return lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


@dataclass
class OracleResult:
    count: int
    calls: int
    memory_bytes: int
    filter_ok: bool
    candidates: list          # per query vertex, sorted uint32 data ids
    tables: dict              # (a, b) -> (off, adj)
    order: np.ndarray
    pivot: np.ndarray
    embeddings: np.ndarray    # [n_emb, q] data ids in query-vertex order
    depth_nodes: np.ndarray = None  # per depth: partial embeddings accepted
    depth_cands: np.ndarray = None  # per depth: candidates examined
    depth_bytes: np.ndarray = None  # per depth: algorithmic bytes of table rows read


class OracleGraph:
    def __init__(self, g):
        self._keep = (np.ascontiguousarray(g.off, np.uint32), np.ascontiguousarray(g.nbr, np.uint32),
                      np.ascontiguousarray(g.labels, np.uint32))
        off, nbr, lab = self._keep
        self.h = _lib().orc_graph_new(_p(off), _p(nbr), _p(lab), g.num_vertices)

    def __del__(self):
        if getattr(self, "h", None):
            _lib().orc_graph_free(self.h)
            self.h = None

    def run(self, q, filter="GQL", order="GQL", cap=0, emit_limit=0, want_tables=True) -> OracleResult:
        lib = _lib()
        qoff = np.ascontiguousarray(q.off, np.uint32)
        qnbr = np.ascontiguousarray(q.nbr, np.uint32)
        qlab = np.ascontiguousarray(q.labels, np.uint32)
        n = q.num_vertices
        r = lib.orc_run(self.h, _p(qoff), _p(qnbr), _p(qlab), n, FILTERS[filter], ORDERS[order], cap, emit_limit)
        try:
            cands = []
            for u in range(n):
                c = np.empty(lib.orc_res_cand_count(r, u), np.uint32)
                if c.size:
                    lib.orc_res_cands(r, u, _p(c))
                cands.append(c)
            tables = {}
            if want_tables:
                for a in range(n):
                    for b in q.neighbors(a):
                        nnz = lib.orc_res_table_nnz(r, a, int(b))
                        off = np.empty(len(cands[a]) + 1, np.uint32)
                        adj = np.empty(max(nnz, 1), np.uint32)
                        lib.orc_res_table(r, a, int(b), _p(off), _p(adj))
                        tables[(a, int(b))] = (off, adj[:nnz])
            order_ = np.empty(n, np.uint32)
            pivot = np.empty(n, np.uint32)
            lib.orc_res_order(r, _p(order_), _p(pivot))
            ne = lib.orc_res_num_emb(r)
            emb = np.empty((ne, n), np.uint32)
            if ne:
                lib.orc_res_emb(r, _p(emb))
            stats = [np.zeros(n, np.uint64) for _ in range(3)]
            lib.orc_res_depth_stats(r, *[a.ctypes.data_as(C.POINTER(C.c_uint64)) for a in stats])
            return OracleResult(count=int(lib.orc_res_count(r)), calls=int(lib.orc_res_calls(r)),
                                memory_bytes=int(lib.orc_res_memory(r)), filter_ok=bool(lib.orc_res_filter_ok(r)),
                                candidates=cands, tables=tables, order=order_, pivot=pivot, embeddings=emb,
                                depth_nodes=stats[0], depth_cands=stats[1], depth_bytes=stats[2])
        finally:
            lib.orc_res_free(r)


def parse_ref_dump(text: str):
    """Parses the line format printed by tests/golden/ref_dump.cpp."""
    cands, tables, order, pivot, mem = {}, {}, None, None, None
    for line in text.splitlines():
        p = line.split()
        if not p:
            continue
        if p[0] == "C":
            u, n = int(p[1]), int(p[2])
            cands[u] = np.array(p[3:3 + n], dtype=np.uint32)
        elif p[0] == "T":
            a, b, nnz = int(p[1]), int(p[2]), int(p[3])
            bar = p.index("|")
            tables[(a, b)] = (np.array(p[4:bar], dtype=np.uint32), np.array(p[bar + 1:], dtype=np.uint32))
            assert len(tables[(a, b)][1]) == nnz
        elif p[0] == "O":
            order = np.array(p[1:], dtype=np.uint32)
        elif p[0] == "P":
            pivot = np.array(p[1:], dtype=np.uint32)
        elif p[0] == "M":
            mem = int(p[1])
    return {"cands": [cands[u] for u in sorted(cands)], "tables": tables, "order": order, "pivot": pivot,
            "memory": mem}
