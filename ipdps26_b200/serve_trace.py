"""Request traces for the served workload and their replay.

A trace is a list of requests with Poisson arrival times over a set of
resident graphs: update batches (log-uniform edit counts, a fixed insert
fraction, deletions drawn uniformly from the graph's live ids at that point
of the trace) and full-count queries. Each graph's ids are followed with the
rule hm_graph_apply_batch and the server use (deleted ids are freed, then
insertions take the smallest free ids, then new ones), so every deletion in
the trace names a live hyperedge when it is served in arrival order.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import engine, gen


@dataclass
class Request:
    t: float                 # arrival, seconds after the start of the replay
    graph: int
    kind: int                # engine.REQ_UPDATE or engine.REQ_COUNT
    dels: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    ins_off: np.ndarray = field(default_factory=lambda: np.zeros(1, np.uint64))
    ins_mem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    ids: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))  # ids its insertions get

    @property
    def edits(self) -> int:
        return len(self.dels) + len(self.ins_off) - 1


class IdMirror:
    """Live ids of one graph under smallest-free-first assignment."""

    def __init__(self, n_edges: int):
        self.live = np.ones(n_edges, bool)

    def live_ids(self) -> np.ndarray:
        return np.flatnonzero(self.live).astype(np.uint32)

    def apply(self, dels: np.ndarray, n_ins: int) -> np.ndarray:
        self.live[dels] = False
        free = np.flatnonzero(~self.live)[:n_ins]
        extra = n_ins - len(free)
        new = np.arange(len(self.live), len(self.live) + extra)
        if extra:
            self.live = np.concatenate([self.live, np.zeros(extra, bool)])
        ids = np.concatenate([free, new]).astype(np.uint32)
        self.live[ids] = True
        return ids


def make_trace(graph_params, rate: float, duration: float, seed: int, update_fraction: float = 0.7,
               edits_min: int = 100, edits_max: int = 10_000, insert_fraction: float = 0.8,
               max_requests: int | None = None) -> list[Request]:
    """Poisson arrivals at `rate` per second for `duration` seconds; each
    request picks a graph uniformly, then is an update with probability
    `update_fraction` (else a full count)."""
    rng = np.random.default_rng(seed)
    mirrors = [IdMirror(p.n_edges) for p in graph_params]
    out: list[Request] = []
    t = 0.0
    lo, hi = np.log(edits_min), np.log(edits_max)
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and len(out) >= max_requests):
            break
        g = int(rng.integers(len(graph_params)))
        if rng.random() < update_fraction:
            n_edits = int(round(np.exp(rng.uniform(lo, hi))))
            dels, ins = gen.batch(graph_params[g], int(rng.integers(1 << 62)), mirrors[g].live_ids(), n_edits,
                                  insert_fraction)
            ids = mirrors[g].apply(dels, ins.n_edges)
            out.append(Request(t, g, engine.REQ_UPDATE, dels, ins.offsets, ins.members, ids))
        else:
            out.append(Request(t, g, engine.REQ_COUNT))
    return out


@dataclass
class Replay:
    results: list            # per request: (ServeResult, assigned ids)
    wall_s: float            # first arrival to last completion
    submit_lag_ms: float     # worst lateness of a submission against its arrival time


def replay(server: "engine.Server", trace: list[Request], paced: bool = True) -> Replay:
    """Submits the trace at its arrival times (or all at once), waits for
    every result. Latencies come from the server's own clock."""
    tickets = [0] * len(trace)
    lag = 0.0
    t0 = time.perf_counter()
    for i, r in enumerate(trace):
        if paced:
            d = r.t - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            lag = max(lag, (time.perf_counter() - t0) - r.t)
        if r.kind == engine.REQ_UPDATE:
            tickets[i] = server.submit_update(r.graph, r.dels, r.ins_off, r.ins_mem)
        else:
            tickets[i] = server.submit_count(r.graph)
    server.drain()
    wall = time.perf_counter() - t0
    cap = max([len(r.ins_off) - 1 for r in trace] + [1])
    results = [server.wait(t, cap) for t in tickets]
    return Replay(results, wall, 1000.0 * lag)


def summarize(trace: list[Request], rep: Replay) -> dict:
    """Latency percentiles and throughput of one replay (server clock)."""
    res = [r for r, _ in rep.results]
    lat = np.array([r.done_ms - r.submit_ms for r in res])
    upd = np.array([r.kind == engine.REQ_UPDATE for r in res])
    first = min(r.submit_ms for r in res)
    last = max(r.done_ms for r in res)
    span_s = (last - first) / 1000.0
    edits = sum(t.edits for t in trace if t.kind == engine.REQ_UPDATE)
    rounds = np.array([r.round_requests for r in res])

    def pct(x, q):
        return float(np.percentile(x, q)) if len(x) else None

    return {
        "requests": len(res), "updates": int(upd.sum()), "counts": int((~upd).sum()),
        "failed": int(sum(r.status != 0 for r in res)),
        "span_s": span_s, "update_batches_per_s": float(upd.sum()) / span_s, "requests_per_s": len(res) / span_s,
        "edits_per_s": edits / span_s,
        "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
        "update_p50_ms": pct(lat[upd], 50), "update_p99_ms": pct(lat[upd], 99),
        "count_p50_ms": pct(lat[~upd], 50), "count_p99_ms": pct(lat[~upd], 99),
        "mean_round_requests": float(rounds.mean()) if len(rounds) else 0.0,
        "submit_lag_ms": rep.submit_lag_ms,
    }


def same_results(a: Replay, b: Replay) -> bool:
    """Bit-exact agreement of two replays of one trace (ids, deltas, counts)."""
    for (ra, ia), (rb, ib) in zip(a.results, b.results):
        if ra.status != rb.status or ra.kind != rb.kind or not np.array_equal(ia, ib):
            return False
        if list(ra.delta30) != list(rb.delta30) or list(ra.counts30) != list(rb.counts30):
            return False
    return len(a.results) == len(b.results)


__all__ = ["Request", "IdMirror", "make_trace", "Replay", "replay", "summarize", "same_results"]
