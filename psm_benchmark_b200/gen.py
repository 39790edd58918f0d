"""Seeded synthetic workloads (ctypes front end of libpsm_gen.so).

Workload definitions follow the benchmark configurations of the subgraph
matching path:

  plain_small  Chung-Lu (n=9,460, exponent 2.3, avg degree 7.8), 307 labels
               Zipf(1.1); 200 random-walk queries of 8 vertices, half sparse
               and half dense; GQL filter + GQL order, no cap.
  plain_rmat   R-MAT scale 20 (a=.57, b=c=.19, edge factor 8), 32 uniform
               labels; 100 queries each of 12 and 16 vertices; CFL filter +
               CFL order, cap 1e9.
  batched      same graph as plain_rmat; 2,000 queries, sizes uniform over
               {4,6,8,12,16,24,32}.
  join         R-MAT scale 22, edge factor 16, 64 Zipf(1.0) labels; 200 queries
               of 24..32 vertices, matched by decomposition + hash join.
  serve        R-MAT scale 24, edge factor 16, 128 uniform labels; a Poisson
               stream of queries with sizes {4,8,12,16,24,32} weighted
               .3/.25/.2/.1/.1/.05.

Seeds: workload index i uses 0x50534D00 + i; query j uses that seed xor j.
Sparse/dense alternates by query index (even = sparse, odd = dense).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from functools import lru_cache
from pathlib import Path

import numpy as np

from .graphs import Graph

_PKG = Path(__file__).resolve().parent


class _Csr(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_entries", C.c_uint64),
                ("off", C.POINTER(C.c_uint32)), ("nbr", C.POINTER(C.c_uint32))]


@lru_cache(maxsize=1)
def _lib():
    path = _PKG / "libpsm_gen.so"
    if not path.exists():
        from .build import build_gen
        build_gen()
    lib = C.CDLL(str(path))
    u32p = C.POINTER(C.c_uint32)
    lib.psmgen_chung_lu.argtypes = [C.c_uint32, C.c_double, C.c_double, C.c_uint64, C.POINTER(_Csr)]
    lib.psmgen_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                C.c_uint64, C.POINTER(_Csr)]
    lib.psmgen_labels.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, u32p]
    lib.psmgen_query.argtypes = [u32p, u32p, u32p, C.c_uint32, C.c_uint32, C.c_int, C.c_uint64,
                                 u32p, u32p, C.c_uint32, u32p, u32p]
    lib.psmgen_free.argtypes = [C.c_void_p]
    lib.psmgen_write_text.argtypes = [u32p, u32p, u32p, C.c_uint32, C.c_char_p]
    lib.psmgen_write_text.restype = C.c_int
    for f in (lib.psmgen_chung_lu, lib.psmgen_rmat, lib.psmgen_labels, lib.psmgen_query):
        f.restype = C.c_int
    return lib


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _take_csr(c: _Csr):
    lib = _lib()
    n = c.num_vertices
    off = np.ctypeslib.as_array(c.off, shape=(n + 1,)).copy()
    nnz = int(c.num_entries)
    nbr = np.ctypeslib.as_array(c.nbr, shape=(max(nnz, 1),))[:nnz].copy()
    lib.psmgen_free(C.cast(c.off, C.c_void_p))
    lib.psmgen_free(C.cast(c.nbr, C.c_void_p))
    return off, nbr


def chung_lu(n: int, gamma: float, avg_degree: float, seed: int):
    c = _Csr()
    rc = _lib().psmgen_chung_lu(n, gamma, avg_degree, seed, C.byref(c))
    if rc:
        raise RuntimeError(f"psmgen_chung_lu failed ({rc})")
    return _take_csr(c)


def rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int):
    cs = _Csr()
    rc = _lib().psmgen_rmat(scale, edge_factor, a, b, c, seed, C.byref(cs))
    if rc:
        raise RuntimeError(f"psmgen_rmat failed ({rc})")
    return _take_csr(cs)


def labels(n: int, num_labels: int, zipf_s: float, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    rc = _lib().psmgen_labels(n, num_labels, zipf_s, seed, _u32p(out))
    if rc:
        raise RuntimeError(f"psmgen_labels failed ({rc})")
    return out


def query(g: Graph, k: int, dense: bool, seed: int) -> Graph:
    """Random-walk query of k vertices taken from g (always has an embedding)."""
    ql = np.empty(k, dtype=np.uint32)
    maxe = k * (k - 1) // 2 + 1
    edges = np.empty(2 * maxe, dtype=np.uint32)
    ne = np.zeros(1, dtype=np.uint32)
    rc = _lib().psmgen_query(_u32p(g.off), _u32p(g.nbr), _u32p(g.labels), g.num_vertices, k,
                             1 if dense else 0, seed & 0xFFFFFFFFFFFFFFFF, _u32p(ql), _u32p(edges),
                             maxe, _u32p(ne), None)
    if rc:
        raise RuntimeError(f"psmgen_query failed ({rc})")
    m = int(ne[0])
    return Graph.from_edges(k, ql, edges[: 2 * m].reshape(-1, 2))


def write_text(g: Graph, path) -> None:
    """Fast writer of the reference text format (same output as Graph.write_text)."""
    off = np.ascontiguousarray(g.off, np.uint32)
    nbr = np.ascontiguousarray(g.nbr, np.uint32)
    lab = np.ascontiguousarray(g.labels, np.uint32)
    rc = _lib().psmgen_write_text(_u32p(off), _u32p(nbr), _u32p(lab), g.num_vertices, str(path).encode())
    if rc:
        raise RuntimeError(f"psmgen_write_text failed ({rc})")


BASE_SEED = 0x50534D00


@dataclass
class Workload:
    name: str
    index: int
    graph: Graph
    queries: list = field(default_factory=list)
    filter: str = "CFL"
    order: str = "CFL"
    engine: str = "EXPLORE"
    cap: int = 0            # 0 = no cap

    @property
    def method(self) -> str:
        return f"{self.filter}_{self.order}_{self.engine}"

    @property
    def seed(self) -> int:
        return BASE_SEED + self.index


def make_graph(kind: str, index: int, scale: int = 0, edge_factor: int = 0, n: int = 0,
               num_labels: int = 32, zipf_s: float = 0.0) -> Graph:
    seed = BASE_SEED + index
    if kind == "chung_lu":
        off, nbr = chung_lu(n, 2.3, 7.8, seed)
    else:
        off, nbr = rmat(scale, edge_factor, 0.57, 0.19, 0.19, seed)
    lab = labels(off.shape[0] - 1, num_labels, zipf_s, seed)
    return Graph(off=off, nbr=nbr, labels=lab)


def make_queries(g: Graph, sizes, seed: int, start_id: int = 0):
    out = []
    for j, k in enumerate(sizes):
        qid = start_id + j
        out.append(query(g, int(k), dense=(qid % 2 == 1), seed=seed ^ qid))
    return out


def plain_small(num_queries: int = 200) -> Workload:
    g = make_graph("chung_lu", 1, n=9460, num_labels=307, zipf_s=1.1)
    w = Workload("plain_small", 1, g, filter="GQL", order="GQL", engine="GQL", cap=0)
    w.queries = make_queries(g, [8] * num_queries, w.seed)
    return w


def plain_rmat(num_queries: int = 200, scale: int = 20) -> Workload:
    g = make_graph("rmat", 2, scale=scale, edge_factor=8, num_labels=32)
    w = Workload("plain_rmat", 2, g, filter="CFL", order="CFL", engine="EXPLORE", cap=10**9)
    half = num_queries // 2
    w.queries = make_queries(g, [12] * half + [16] * (num_queries - half), w.seed)
    return w


def batched_sizes(num_queries: int, seed: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.choice(np.array([4, 6, 8, 12, 16, 24, 32]), size=num_queries)


def batched(num_queries: int = 2000, scale: int = 20, graph: Graph | None = None) -> Workload:
    g = graph if graph is not None else make_graph("rmat", 2, scale=scale, edge_factor=8, num_labels=32)
    w = Workload("batched", 3, g, filter="CFL", order="CFL", engine="EXPLORE", cap=10**9)
    w.queries = make_queries(g, batched_sizes(num_queries, w.seed), w.seed)
    return w


SERVE_SIZES = np.array([4, 8, 12, 16, 24, 32])
SERVE_WEIGHTS = np.array([0.3, 0.25, 0.2, 0.1, 0.1, 0.05])


def serve_sizes(num_queries: int, seed: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.choice(SERVE_SIZES, size=num_queries, p=SERVE_WEIGHTS)


def join_sizes(num_queries: int, seed: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.integers(24, 33, size=num_queries)


def join(num_queries: int = 200, scale: int = 22, graph: Graph | None = None) -> Workload:
    """Decomposition + hash join: R-MAT scale 22, edge factor 16, 64
    Zipf(1.0) labels; 24..32-vertex queries, joined from units of <= 12
    vertices."""
    g = graph if graph is not None else make_graph("rmat", 4, scale=scale, edge_factor=16, num_labels=64,
                                                   zipf_s=1.0)
    w = Workload("join", 4, g, filter="CFL", order="CFL", engine="EXPLORE", cap=0)
    w.queries = make_queries(g, join_sizes(num_queries, w.seed), w.seed)
    return w


def serve(num_queries: int = 50000, scale: int = 24, graph: Graph | None = None) -> Workload:
    """Serving: R-MAT scale 24, edge factor 16, 128 uniform labels; query sizes
    {4,8,12,16,24,32} weighted .3/.25/.2/.1/.1/.05; cap 1e9."""
    g = graph if graph is not None else make_graph("rmat", 5, scale=scale, edge_factor=16, num_labels=128)
    w = Workload("serve", 5, g, filter="CFL", order="CFL", engine="EXPLORE", cap=10**9)
    w.queries = make_queries(g, serve_sizes(num_queries, w.seed), w.seed)
    return w


def poisson_arrivals(num: int, rate_per_s: float, seed: int) -> np.ndarray:
    """Arrival times (s) of a Poisson stream of `num` requests."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=num))
