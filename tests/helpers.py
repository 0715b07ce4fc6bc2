"""Shared test utilities: golden fixtures and graph regeneration."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_golden(kind: str) -> dict:
    return json.loads((GOLDEN / f"{kind}_golden.json").read_text())


def digest(h) -> str:
    m = hashlib.sha256()
    m.update(np.ascontiguousarray(h.offsets, np.uint64).tobytes())
    m.update(np.ascontiguousarray(h.members, np.uint32).tobytes())
    if h.timestamps is not None:
        m.update(np.ascontiguousarray(h.timestamps, np.int64).tobytes())
    return m.hexdigest()


def static_case(p: dict):
    from ipdps26_b200 import gen

    kw = dict(p)
    dedupe = kw.pop("dedupe", True)
    return gen.static(gen.params(dedupe=dedupe, **kw))


def temporal_case(c: dict):
    from ipdps26_b200 import gen

    kw = dict(c["gen"])
    dedupe = kw.pop("dedupe", False)
    return gen.temporal(gen.params(dedupe=dedupe, **kw), **c["burst"])


def csr(rows):
    """CSR arrays from a list of member lists."""
    off = [0]
    mem = []
    for r in rows:
        mem.extend(r)
        off.append(len(mem))
    return np.array(off, np.uint64), np.array(mem, np.uint32)


def random_graph(rng, n_edges, n_nodes, kmax, p_repeat=0.0):
    """Small random hypergraph as (offsets, members) with unsorted rows and,
    optionally, repeated node ids inside rows (both are legal inputs)."""
    rows = []
    for _ in range(n_edges):
        k = int(rng.integers(1, kmax + 1))
        r = list(rng.choice(n_nodes, size=min(k, n_nodes), replace=False))
        if p_repeat and rng.random() < p_repeat:
            r.append(r[0])
        rng.shuffle(r)
        rows.append(r)
    return csr(rows)
