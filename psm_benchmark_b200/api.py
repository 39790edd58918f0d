"""Python host API over the C ABI, mirroring the reference's operator
surface: a data graph resident on the device, one call per query that runs
filter -> tables -> order -> enumerate with a "FILTER_ORDER_ENGINE" method
string (the reference's -BackMethods triple), an embedding cap (-num) and a
time limit (-time_limit), plus the batched path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native as N
from .graphs import Graph


def _u32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


class Engine:
    """A device context: one CUDA stream and one device arena."""

    def __init__(self, device: int = 0, arena_bytes: int = 4 << 30):
        self._h = C.c_void_p()
        N.check(N.lib().psm_context_create(device, arena_bytes, C.byref(self._h)))

    def close(self):
        if self._h:
            N.lib().psm_context_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class DataGraph:
    """Data graph uploaded to HBM as a label-major CSR."""

    def __init__(self, h):
        self._h = h

    @classmethod
    def from_graph(cls, g: Graph) -> "DataGraph":
        off = np.ascontiguousarray(g.off, np.uint32)
        nbr = np.ascontiguousarray(g.nbr, np.uint32)
        lab = np.ascontiguousarray(g.labels, np.uint32)
        h = C.c_void_p()
        N.check(N.lib().psm_graph_from_csr(_u32p(off), _u32p(nbr), _u32p(lab), g.num_vertices, C.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path) -> "DataGraph":
        h = C.c_void_p()
        N.check(N.lib().psm_graph_load(str(path).encode(), C.byref(h)))
        return cls(h)

    def info(self):
        V, L, md, mf = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        E = C.c_uint64()
        N.check(N.lib().psm_graph_info(self._h, C.byref(V), C.byref(E), C.byref(L), C.byref(md), C.byref(mf)))
        return {"vertices": V.value, "edges": E.value, "labels": L.value, "max_degree": md.value,
                "max_label_frequency": mf.value}

    def close(self):
        if self._h:
            N.lib().psm_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _QueryBuf:
    """Keeps the numpy arrays of a query descriptor alive."""

    def __init__(self, q: Graph):
        self.labels = np.ascontiguousarray(q.labels, np.uint32)
        self.edges = np.ascontiguousarray(q.edge_list().astype(np.uint32).reshape(-1))
        self.desc = N.QueryDesc(q.num_vertices, len(self.edges) // 2, _u32p(self.labels), _u32p(self.edges))


def options(method: str = "CFL_CFL_EXPLORE", cap: int = 0, time_limit: float = 60.0, emit: int = 0) -> N.Options:
    f, o, e = N.parse_method(method)
    return N.Options(f, o, e, 1 if emit else 0, int(cap), float(time_limit), int(emit))


@dataclass
class MatchResult:
    count: int
    calls: int
    memory_bytes: int
    table_entries: int
    alg_bytes: int
    donations: int
    overtime: bool
    filter_ok: bool
    status: int
    prep_ms: float
    enum_ms: float
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    tasks: int = 0
    idle_polls: int = 0

    @staticmethod
    def of(r: N.Result) -> "MatchResult":
        return MatchResult(count=r.count, calls=r.calls, memory_bytes=r.memory_bytes, table_entries=r.table_entries,
                           alg_bytes=r.alg_bytes, donations=r.donations, overtime=bool(r.overtime),
                           filter_ok=bool(r.filter_ok), status=r.status, prep_ms=r.prep_ms, enum_ms=r.enum_ms,
                           h2d_bytes=r.h2d_bytes, d2h_bytes=r.d2h_bytes, tasks=r.tasks, idle_polls=r.idle_polls)


def match(engine: Engine, data: DataGraph, query: Graph, method: str = "CFL_CFL_EXPLORE", cap: int = 0,
          time_limit: float = 60.0) -> MatchResult:
    """Plain path: one query, the whole GPU."""
    qb = _QueryBuf(query)
    opt = options(method, cap, time_limit)
    res = N.Result()
    N.check(N.lib().psm_match(engine._h, data._h, C.byref(qb.desc), C.byref(opt), C.byref(res)),
            allow=(N.PSM_ERR_TIMEOUT,))
    return MatchResult.of(res)


def match_batch(engine: Engine, data: DataGraph, queries, method: str = "CFL_CFL_EXPLORE", cap: int = 0,
                time_limit: float = 60.0):
    """Batched path: all queries through one preparation launch and one
    enumeration launch."""
    bufs = [_QueryBuf(q) for q in queries]
    arr = (N.QueryDesc * len(bufs))(*[b.desc for b in bufs])
    opt = options(method, cap, time_limit)
    res = (N.Result * len(bufs))()
    N.check(N.lib().psm_match_batch(engine._h, data._h, arr, len(bufs), C.byref(opt), res),
            allow=(N.PSM_ERR_TIMEOUT,))
    return [MatchResult.of(r) for r in res]


class Run:
    """A finished plain-path query whose device state can be inspected
    (candidates, tables, order, embeddings). One live Run per Engine."""

    def __init__(self, engine: Engine, data: DataGraph, query: Graph, method: str = "CFL_CFL_EXPLORE",
                 cap: int = 0, time_limit: float = 60.0, emit: int = 0):
        self.query = query
        qb = _QueryBuf(query)
        opt = options(method, cap, time_limit, emit)
        self._h = C.c_void_p()
        res = N.Result()
        N.check(N.lib().psm_run_create(engine._h, data._h, C.byref(qb.desc), C.byref(opt), C.byref(self._h),
                                       C.byref(res)), allow=(N.PSM_ERR_TIMEOUT,))
        self.result = MatchResult.of(res)

    def candidates(self, u: int) -> np.ndarray:
        n = C.c_uint32()
        N.check(N.lib().psm_run_candidates(self._h, u, None, 0, C.byref(n)))
        out = np.empty(n.value, np.uint32)
        N.check(N.lib().psm_run_candidates(self._h, u, _u32p(out), n.value, C.byref(n)))
        return out

    def table(self, a: int, b: int):
        rows, nnz = C.c_uint32(), C.c_uint32()
        N.check(N.lib().psm_run_table(self._h, a, b, None, 0, None, 0, C.byref(rows), C.byref(nnz)))
        off = np.empty(rows.value + 1, np.uint32)
        adj = np.empty(max(nnz.value, 1), np.uint32)
        N.check(N.lib().psm_run_table(self._h, a, b, _u32p(off), len(off), _u32p(adj), len(adj), C.byref(rows),
                                      C.byref(nnz)))
        return off, adj[: nnz.value]

    def order(self):
        n = self.query.num_vertices
        o = np.empty(n, np.uint32)
        p = np.empty(n, np.uint32)
        N.check(N.lib().psm_run_order(self._h, _u32p(o), _u32p(p)))
        return o, p

    def embeddings(self) -> np.ndarray:
        rows = C.c_uint64()
        N.check(N.lib().psm_run_embeddings(self._h, None, 0, C.byref(rows)))
        out = np.empty((rows.value, self.query.num_vertices), np.uint32)
        if rows.value:
            N.check(N.lib().psm_run_embeddings(self._h, _u32p(out), rows.value, C.byref(rows)))
        return out

    def close(self):
        if self._h:
            N.lib().psm_run_free(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
