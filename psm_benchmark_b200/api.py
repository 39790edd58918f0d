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

    def batch_tuning(self) -> dict:
        """Settings of this context's batched launches (the intersection
        variant applies to every enumeration launch of the context)."""
        t = N.BatchTuning()
        N.check(N.lib().psm_context_get_batch_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_batch_tuning(self, team: str = "RULE", grabs_per_warp: int = 8, enum_quarters: int = 4,
                         intersect: str = "BINARY"):
        t = N.BatchTuning(N.TEAMS[team], int(grabs_per_warp), int(enum_quarters), N.INTERSECTS[intersect], 0.0)
        N.check(N.lib().psm_context_set_batch_tuning(self._h, C.byref(t)))

    def autotune_batch(self, data, queries, method: str = "CFL_CFL_EXPLORE", cap: int = 0,
                       time_limit: float = 60.0, repeats: int = 2) -> dict:
        """Times the sample batch under every candidate setting, installs the
        fastest in this context. Returns {"best": ..., "tried": [...]}."""
        bufs = [_QueryBuf(q) for q in queries]
        arr = (N.QueryDesc * len(bufs))(*[b.desc for b in bufs])
        opt = options(method, cap, time_limit)
        best = N.BatchTuning()
        tried = (N.BatchTuning * 32)()
        nt = C.c_uint32()
        N.check(N.lib().psm_autotune_batch(self._h, data._h, arr, len(bufs), C.byref(opt), int(repeats),
                                           C.byref(best), tried, 32, C.byref(nt)))
        return {"best": best.as_dict(), "tried": [tried[i].as_dict() for i in range(nt.value)]}

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

    @classmethod
    def load_binary(cls, prefix) -> "DataGraph":
        """Reference binary format: <prefix>_deg.bin, _adj.bin, _label.bin."""
        h = C.c_void_p()
        N.check(N.lib().psm_graph_load_binary(f"{prefix}_deg.bin".encode(), f"{prefix}_adj.bin".encode(),
                                              f"{prefix}_label.bin".encode(), C.byref(h)))
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
    count_internal: int = 0  # unclamped count: the work alg_bytes covers

    @staticmethod
    def of(r: N.Result) -> "MatchResult":
        return MatchResult(count=r.count, calls=r.calls, memory_bytes=r.memory_bytes, table_entries=r.table_entries,
                           alg_bytes=r.alg_bytes, donations=r.donations, overtime=bool(r.overtime),
                           filter_ok=bool(r.filter_ok), status=r.status, prep_ms=r.prep_ms, enum_ms=r.enum_ms,
                           h2d_bytes=r.h2d_bytes, d2h_bytes=r.d2h_bytes, tasks=r.tasks, idle_polls=r.idle_polls,
                           count_internal=r.count_internal)


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


# ------------------------------------------------------------- join path --

@dataclass
class JoinResult:
    count: int
    units: list            # vertex masks of the decomposition units
    unit_rows: list        # embeddings of each unit
    join_rows: list        # rows after joining units 0..k
    prep_ms: float
    enum_ms: float
    join_ms: float
    work_bytes: int
    memory_bytes: int


def match_join(engine: Engine, data: DataGraph, query: Graph, method: str = "CFL_CFL_EXPLORE",
               max_unit_vertices: int = 12, cap: int = 0, time_limit: float = 60.0, pattern: str = "BOUNDED",
               join_method: str = "LEFTDEEP") -> JoinResult:
    """Decomposition + hash-join path: the query is filtered and tabled
    whole, split into units (pattern: BOUNDED = connected units of at most
    max_unit_vertices vertices; the reference's STAR, TWINTWIG, SEED,
    SKETCHTREE; COST = bounded units of least estimated cost), each unit's
    embeddings are materialised on the device and joined on shared query
    vertices, left-deep or bushy."""
    qb = _QueryBuf(query)
    opt = options(method, cap, time_limit)
    jo = N.JoinOptions(N.SPLIT_PATTERNS[pattern], N.JOIN_METHODS[join_method], int(max_unit_vertices), 0)
    r = N.JoinResult()
    N.check(N.lib().psm_match_join_ex(engine._h, data._h, C.byref(qb.desc), C.byref(opt), C.byref(jo), C.byref(r)))
    u = r.units
    return JoinResult(count=r.count, units=list(r.unit_mask[:u]), unit_rows=list(r.unit_rows[:u]),
                      join_rows=list(r.join_rows[:u]), prep_ms=r.prep_ms, enum_ms=r.enum_ms, join_ms=r.join_ms,
                      work_bytes=r.work_bytes, memory_bytes=r.memory_bytes)


def decompose(query: Graph, max_unit_vertices: int = 12) -> list:
    """Vertex masks of the units psm_match_join uses (host only)."""
    qb = _QueryBuf(query)
    n = C.c_uint32()
    masks = (C.c_uint32 * N.MAX_UNITS)()
    N.check(N.lib().psm_query_decompose(C.byref(qb.desc), int(max_unit_vertices), C.byref(n), masks))
    return list(masks[: n.value])


def join_plan(query: Graph, pattern: str = "BOUNDED", join_method: str = "LEFTDEEP", max_unit_vertices: int = 12,
              data_vertices: float = 1e6, data_edges: float = 8e6):
    """The units and binary joins psm_match_join_ex would use (host only; the
    cost searches use the label-blind card model of a data graph with the
    given sizes). Returns (unit masks, [(left, right), ...]): operands are
    unit indices, or len(units) + i for the result of join i."""
    qb = _QueryBuf(query)
    jo = N.JoinOptions(N.SPLIT_PATTERNS[pattern], N.JOIN_METHODS[join_method], int(max_unit_vertices), 0)
    n, nj = C.c_uint32(), C.c_uint32()
    masks = (C.c_uint32 * N.MAX_UNITS)()
    ops = (C.c_uint32 * (4 * N.MAX_UNITS))()
    N.check(N.lib().psm_query_decompose_ex(C.byref(qb.desc), C.byref(jo), float(data_vertices), float(data_edges),
                                           C.byref(n), masks, C.byref(nj), ops))
    return list(masks[: n.value]), [(ops[2 * j], ops[2 * j + 1]) for j in range(nj.value)]


def hash_join(engine: Engine, r_rows: np.ndarray, r_vertex, s_rows: np.ndarray, s_vertex, vertex_label=None,
              count_only: bool = False):
    """One device hash join of host relations (R builds, S probes). Returns
    (rows, out_vertex) or, with count_only, the number of rows."""
    R = np.ascontiguousarray(r_rows, np.uint32).reshape(len(r_rows), len(r_vertex))
    S = np.ascontiguousarray(s_rows, np.uint32).reshape(len(s_rows), len(s_vertex))
    rv = np.ascontiguousarray(r_vertex, np.uint32)
    sv = np.ascontiguousarray(s_vertex, np.uint32)
    lab = None if vertex_label is None else np.ascontiguousarray(vertex_label, np.uint32)
    labp = _u32p(lab) if lab is not None else None
    n = C.c_uint64()
    L = N.lib()
    N.check(L.psm_hash_join(engine._h, _u32p(R), R.shape[0], R.shape[1], _u32p(rv), _u32p(S), S.shape[0], S.shape[1],
                            _u32p(sv), labp, None, 0, None, None, C.byref(n)))
    if count_only:
        return n.value
    total = n.value
    ov = np.zeros(32, np.uint32)
    oc = C.c_uint32()
    out = np.empty((max(total, 1), 32), np.uint32)
    N.check(L.psm_hash_join(engine._h, _u32p(R), R.shape[0], R.shape[1], _u32p(rv), _u32p(S), S.shape[0], S.shape[1],
                            _u32p(sv), labp, _u32p(out), total, _u32p(ov), C.byref(oc), C.byref(n)))
    w = oc.value
    rows = np.frombuffer(out.tobytes()[: total * w * 4], np.uint32).reshape(total, w) if total else \
        np.empty((0, w), np.uint32)
    return rows, list(ov[:w])


# --------------------------------------------------------------- serving --

@dataclass
class RequestResult:
    ticket: int
    count: int
    status: int
    overtime: bool
    submit_ns: int
    start_ns: int
    done_ns: int
    batch_size: int
    lane: int
    prep_ms: float
    enum_ms: float

    @property
    def latency_ms(self) -> float:
        return (self.done_ns - self.submit_ns) / 1e6


class Server:
    """Request loop over a resident data graph with continuous batching:
    `lanes` batches run side by side, each admitting the queued requests
    that fit its device-memory budget when it frees up."""

    def __init__(self, data: DataGraph, method: str = "CFL_CFL_EXPLORE", cap: int = 0, time_limit: float = 60.0,
                 lanes: int = 2, max_batch: int = 256, lane_arena_bytes: int = 8 << 30, full_gpu_lanes: bool = False,
                 device: int = 0):
        self.data = data  # keeps the graph alive
        opt = options(method, cap, time_limit)
        cfg = N.ServerConfig(lanes, max_batch, lane_arena_bytes, 1 if full_gpu_lanes else 0, 0)
        self._h = C.c_void_p()
        N.check(N.lib().psm_server_create(device, data._h, C.byref(opt), C.byref(cfg), C.byref(self._h)))

    @staticmethod
    def clock_ns() -> int:
        return N.lib().psm_server_clock_ns()

    def submit(self, query: Graph) -> int:
        qb = _QueryBuf(query)
        t = C.c_uint64()
        N.check(N.lib().psm_server_submit(self._h, C.byref(qb.desc), C.byref(t)))
        return t.value

    def set_batch_tuning(self, team: str = "RULE", grabs_per_warp: int = 8, enum_quarters: int = 4,
                         intersect: str = "BINARY"):
        """Settings of every lane's batches (as Engine.set_batch_tuning, e.g.
        the best of Engine.autotune_batch), applied before each lane's next batch."""
        t = N.BatchTuning(N.TEAMS[team], int(grabs_per_warp), int(enum_quarters), N.INTERSECTS[intersect], 0.0)
        N.check(N.lib().psm_server_set_batch_tuning(self._h, C.byref(t)))

    def estimate(self, query: Graph):
        qb = _QueryBuf(query)
        b, budget = C.c_uint64(), C.c_uint64()
        N.check(N.lib().psm_server_estimate(self._h, C.byref(qb.desc), C.byref(b), C.byref(budget)))
        return b.value, budget.value

    def poll(self, max_results: int = 4096, wait_s: float = 0.0):
        buf = (N.RequestResult * max_results)()
        n = C.c_uint32()
        N.check(N.lib().psm_server_poll(self._h, buf, max_results, C.byref(n), float(wait_s)))
        return [RequestResult(ticket=r.ticket, count=r.count, status=r.status, overtime=bool(r.overtime),
                              submit_ns=r.submit_ns, start_ns=r.start_ns, done_ns=r.done_ns, batch_size=r.batch_size,
                              lane=r.lane, prep_ms=r.prep_ms, enum_ms=r.enum_ms) for r in buf[: n.value]]

    def pending(self):
        q, r = C.c_uint64(), C.c_uint64()
        N.check(N.lib().psm_server_pending(self._h, C.byref(q), C.byref(r)))
        return q.value, r.value

    def drain(self, n_expected: int, timeout_s: float = 600.0):
        """Polls until n_expected results have arrived (or the timeout)."""
        out = []
        t_end = Server.clock_ns() + int(timeout_s * 1e9)
        while len(out) < n_expected and Server.clock_ns() < t_end:
            out += self.poll(wait_s=0.05)
        return out

    def close(self):
        if self._h:
            N.lib().psm_server_destroy(self._h)
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


# ------------------------------------------------------- graph file formats --

def store_binary(g: Graph, prefix) -> None:
    """Writes g in the reference's binary format (host only)."""
    off = np.ascontiguousarray(g.off, np.uint32)
    nbr = np.ascontiguousarray(g.nbr, np.uint32)
    lab = np.ascontiguousarray(g.labels, np.uint32)
    N.check(N.lib().psm_graph_store_binary(_u32p(off), _u32p(nbr), _u32p(lab), g.num_vertices,
                                           f"{prefix}_deg.bin".encode(), f"{prefix}_adj.bin".encode(),
                                           f"{prefix}_label.bin".encode()))


def convert_text(text_path, prefix) -> None:
    """Text graph -> reference binary files (the reference's GraphConverter)."""
    N.check(N.lib().psm_graph_convert(str(text_path).encode(), str(prefix).encode()))


def convert_edgelist(edge_list_path, prefix, num_labels: int, seed: int = 0) -> None:
    """Edge list ("u v" per line) -> reference binary files (the reference's
    EdgeListConverter), labels uniform over [0, num_labels) from a seeded
    std::mt19937 (host only)."""
    N.check(N.lib().psm_graph_convert_edgelist(str(edge_list_path).encode(), str(prefix).encode(),
                                               int(num_labels), int(seed)))
