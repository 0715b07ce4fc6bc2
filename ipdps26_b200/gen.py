"""Seeded synthetic workloads (host side), as numpy CSR arrays.

The named configurations restate the workload descriptions the engine is
measured on. Sizes follow a truncated power law and members a
Zipf-Mandelbrot popularity law P(rank r) ~ (r + 1 + q)^-s; ``q`` is the
popularity offset (0 = plain Zipf).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import workloads as W
from ._lib import BurstParams, GenParams, HostGraphInfo, check, lib, ptr, vp


@dataclass
class Hypergraph:
    """Host CSR hypergraph: hyperedge e has members[offsets[e]:offsets[e+1]]."""

    offsets: np.ndarray  # uint64, n_edges + 1
    members: np.ndarray  # uint32
    n_nodes: int
    timestamps: np.ndarray | None = None  # int64 per hyperedge, temporal only

    @property
    def n_edges(self) -> int:
        return len(self.offsets) - 1

    def edge(self, e: int) -> np.ndarray:
        return self.members[self.offsets[e] : self.offsets[e + 1]]

    def subgraph(self, n_edges: int) -> "Hypergraph":
        """The first n_edges hyperedges (same node universe)."""
        off = self.offsets[: n_edges + 1].copy()
        mem = self.members[: off[-1]].copy()
        ts = None if self.timestamps is None else self.timestamps[:n_edges].copy()
        return Hypergraph(off, mem, self.n_nodes, ts)


def _take(handle: vp) -> Hypergraph:
    info = HostGraphInfo()
    check(lib.hm_hostgraph_view(handle, C.byref(info)), "hm_hostgraph_view")
    n, m = info.n_edges, info.n_members
    off = np.ctypeslib.as_array(info.offsets, shape=(n + 1,)).copy()
    mem = np.ctypeslib.as_array(info.members, shape=(max(m, 1),))[:m].copy() if m else np.zeros(0, np.uint32)
    ts = None
    if info.timestamps:
        ts = np.ctypeslib.as_array(info.timestamps, shape=(max(n, 1),))[:n].copy()
    nn = info.n_nodes
    lib.hm_hostgraph_free(handle)
    return Hypergraph(off, mem, nn, ts)


def params(seed, n_nodes, n_edges, k_min, k_max, size_exp, pop_exp, pop_offset=0.0, dedupe=True, permute=True):
    return GenParams(seed, n_nodes, n_edges, k_min, k_max, size_exp, pop_exp, pop_offset, int(dedupe), int(permute))


def static(p: GenParams) -> Hypergraph:
    h = vp()
    check(lib.hm_gen_static(C.byref(p), C.byref(h)), "hm_gen_static")
    return _take(h)


def temporal(p: GenParams, burst_rate=1e-4, events_per_burst=50, gap_mean=20.0, span=100_000_000) -> Hypergraph:
    b = BurstParams(burst_rate, events_per_burst, gap_mean, span)
    h = vp()
    check(lib.hm_gen_temporal(C.byref(p), C.byref(b), C.byref(h)), "hm_gen_temporal")
    return _take(h)


def batch(p: GenParams, batch_seed: int, live_ids: np.ndarray, n_edits: int, insert_fraction: float = 0.8):
    """Returns (sorted deleted ids, inserted Hypergraph)."""
    live = np.ascontiguousarray(live_ids, dtype=np.uint32)
    dels = np.zeros(max(n_edits, 1), np.uint32)
    nd = C.c_uint32(0)
    h = vp()
    check(
        lib.hm_gen_batch(C.byref(p), batch_seed, ptr(live, C.c_uint32), len(live), n_edits, insert_fraction,
                         ptr(dels, C.c_uint32), C.byref(nd), C.byref(h)),
        "hm_gen_batch",
    )
    return dels[: nd.value].copy(), _take(h)


# ---- named workloads (parameters in workloads.py) ---------------------------
C2_Q = W.C2_Q
C5_Q = W.C5_Q


def from_laws(L: W.Laws) -> GenParams:
    return params(L.seed, L.n_nodes, L.n_edges, L.k_min, L.k_max, L.size_exp, L.pop_exp, L.q, dedupe=L.dedupe)


def config1(seed: int = 0, n_nodes: int = 10_000, n_edges: int = 20_000, q: float = 0.0) -> GenParams:
    return from_laws(W.CONFIG1.scaled(seed=seed, n_nodes=n_nodes, n_edges=n_edges, q=q))


def config2(seed: int = 1, n_nodes: int = 1_000_000, n_edges: int = 2_000_000, q: float = C2_Q) -> GenParams:
    return from_laws(W.CONFIG2.scaled(seed=seed, n_nodes=n_nodes, n_edges=n_edges, q=q))


def config4(seed: int = 3, n_nodes: int = 200_000, n_edges: int = 500_000, q: float = 0.0) -> GenParams:
    return from_laws(W.CONFIG4.scaled(seed=seed, n_nodes=n_nodes, n_edges=n_edges, q=q))


def config4_temporal(n_edges: int = W.CONFIG4.n_edges) -> Hypergraph:
    """Config 4's event stream (its first n_edges events when smaller: the
    times of a prefix are those of the full stream)."""
    B = W.CONFIG4_BURSTS
    h = temporal(config4(), B.burst_rate, B.events_per_burst, B.gap_mean, B.span)
    return h if n_edges >= h.n_edges else h.subgraph(n_edges)


# Config 5: resident graphs with |E| log-uniform in [1e3, 2e5] (seeds 100 +
# i), n_nodes = |E| / 2, config-1 size law (k^-2.5 on [2, 25]) and Zipf(1.2)
# popularity with the Zipf-Mandelbrot offset q = 1000 of config 2 (with q = 0
# a 200K-edge graph has a hub in about half of its hyperedges and ~1.8e14
# triples sharing one node, hours of exact counting per request).
def config5_graph(i: int, e_min: int = 1000, e_max: int = 200_000, q: float = C5_Q) -> GenParams:
    seed = 100 + i
    u = np.random.default_rng(seed).uniform(np.log(e_min), np.log(e_max))
    n_edges = int(round(np.exp(u)))
    return params(seed, max(n_edges // 2, 2), n_edges, 2, 25, 2.5, 1.2, q)
