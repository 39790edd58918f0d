"""Host-side graph containers and the reference's text graph format.

The text format is the one the reference loader reads
(graph/graph.cpp:92-172, Graph::loadGraphFromFile):

    t <num_vertices> <num_edges>
    v <id> <label> <degree>        (one line per vertex, ascending id)
    e <u> <v>                      (one line per undirected edge)

Vertex lines must precede edge lines and declared degrees must equal the
actual ones; `write_text` always produces such files.
"""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np


@dataclass
class Graph:
    """Undirected vertex-labelled graph as an id-sorted CSR (uint32)."""

    off: np.ndarray      # uint32[V+1]
    nbr: np.ndarray      # uint32[2E], each row ascending
    labels: np.ndarray   # uint32[V]

    @property
    def num_vertices(self) -> int:
        return int(self.off.shape[0] - 1)

    @property
    def num_entries(self) -> int:
        return int(self.off[-1])

    @property
    def num_edges(self) -> int:
        return self.num_entries // 2

    def degree(self, v: int) -> int:
        return int(self.off[v + 1] - self.off[v])

    def neighbors(self, v: int) -> np.ndarray:
        return self.nbr[self.off[v]:self.off[v + 1]]

    def edge_list(self) -> np.ndarray:
        """Undirected edges (u < v) as an int64[E, 2] array."""
        deg = np.diff(self.off.astype(np.int64))
        src = np.repeat(np.arange(self.num_vertices, dtype=np.int64), deg)
        dst = self.nbr.astype(np.int64)
        keep = src < dst
        return np.stack([src[keep], dst[keep]], axis=1)

    @staticmethod
    def from_edges(num_vertices: int, labels, edges) -> "Graph":
        """Builds the CSR of an undirected simple graph from (u, v) pairs."""
        labels = np.ascontiguousarray(labels, dtype=np.uint32)
        e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
        if e.size:
            if np.any(e[:, 0] == e[:, 1]):
                raise ValueError("self-loops are not allowed")
            lo = np.minimum(e[:, 0], e[:, 1])
            hi = np.maximum(e[:, 0], e[:, 1])
            key = np.unique(lo * (1 << 32) + hi)
            lo, hi = key >> 32, key & 0xFFFFFFFF
            src = np.concatenate([lo, hi])
            dst = np.concatenate([hi, lo])
            order = np.lexsort((dst, src))
            src, dst = src[order], dst[order]
        else:
            src = dst = np.zeros(0, dtype=np.int64)
        deg = np.bincount(src, minlength=num_vertices)
        off = np.zeros(num_vertices + 1, dtype=np.uint32)
        np.cumsum(deg, out=off[1:])
        return Graph(off=off, nbr=dst.astype(np.uint32), labels=labels)

    def write_text(self, path) -> None:
        path = Path(path)
        deg = np.diff(self.off.astype(np.int64))
        el = self.edge_list()
        with open(path, "w") as f:
            f.write(f"t {self.num_vertices} {len(el)}\n")
            v = np.arange(self.num_vertices)
            np.savetxt(f, np.stack([v, self.labels.astype(np.int64), deg], axis=1), fmt="v %d %d %d")
            if len(el):
                np.savetxt(f, el, fmt="e %d %d")

    @staticmethod
    def read_text(path) -> "Graph":
        """Reads the reference text format (vertex lines, then edge lines)."""
        labels = None
        edges = []
        with open(path) as f:
            header = f.readline().split()
            if not header or header[0] != "t":
                raise ValueError(f"{path}: missing 't V E' header")
            n = int(header[1])
            labels = np.zeros(n, dtype=np.uint32)
            for line in f:
                p = line.split()
                if not p:
                    continue
                if p[0] == "v":
                    labels[int(p[1])] = int(p[2])
                elif p[0] == "e":
                    edges.append((int(p[1]), int(p[2])))
        return Graph.from_edges(n, labels, edges)
