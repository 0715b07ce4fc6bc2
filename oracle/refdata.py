"""Datasets that ship with the reference, for parity tests (TEST
INFRASTRUCTURE ONLY).

The reference holds two inputs with known outputs:
  MoCHy-master/dblp_graph.txt                         (MoCHy's sample hypergraph)
  THyMe-main/data/email-Enron-full/email-Enron-full.txt
      with THyMe's results at delta = 86,400,000 in
  THyMe-main/results/email-Enron-full_86400000.000000_{thyme,thymeP,dp}.txt
build_ref.sh copies them verbatim into oracle/_ref/data/ (git-ignored, like
the compiled reference programs), so tests find them on machines without the
reference tree; HM_REFERENCE_ROOT, if set, is the other place looked at.
Nothing here is shipped or used by the engine.
"""
from __future__ import annotations

import hashlib
import os
from pathlib import Path

import numpy as np

DATA = Path(__file__).resolve().parent / "_ref" / "data"

FILES = {
    "dblp": "MoCHy-master/dblp_graph.txt",
    "email-Enron": "THyMe-main/data/email-Enron-full/email-Enron-full.txt",
    "email-Enron-thyme": "THyMe-main/results/email-Enron-full_86400000.000000_thyme.txt",
    "email-Enron-thymeP": "THyMe-main/results/email-Enron-full_86400000.000000_thymeP.txt",
    "email-Enron-dp": "THyMe-main/results/email-Enron-full_86400000.000000_dp.txt",
}
ENRON_DELTA = 86_400_000


def path(name: str) -> Path | None:
    """Where the dataset `name` can be read, or None."""
    rel = FILES[name]
    p = DATA / Path(rel).name
    if p.exists():
        return p
    root = os.environ.get("HM_REFERENCE_ROOT")
    if root and (Path(root) / rel).exists():
        return Path(root) / rel
    return None


def sha256(p: Path) -> str:
    return hashlib.sha256(p.read_bytes()).hexdigest()


def _csr(rows):
    off = np.zeros(len(rows) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    mem = np.array([v for r in rows for v in r], np.uint32)
    return off, mem


def read_mochy(p: Path):
    """MoCHy's reader (MoCHy-master/read_data.cpp:8-45): comma-separated
    0-based node ids, one hyperedge per line, a repeated id in a line counted
    once. Returns (offsets, members, n_nodes)."""
    rows = []
    for ln in p.read_text().splitlines():
        if not ln.strip():
            continue
        r = []
        for t in ln.split(","):
            v = int(t)
            if v not in r:
                r.append(v)
        rows.append(r)
    off, mem = _csr(rows)
    return off, mem, int(mem.max()) + 1


def read_thyme(p: Path):
    """THyMe's reader (THyMe-main/code/read_data.cpp:22-57): "n1,n2,...<TAB>t"
    lines with integer times. Returns (offsets, members, times, n_nodes) in
    file order."""
    rows, ts = [], []
    for ln in p.read_text().splitlines():
        if not ln.strip():
            continue
        nodes, t = ln.split("\t")
        r = []
        for x in nodes.split(","):
            v = int(x)
            if v not in r:
                r.append(v)
        rows.append(r)
        ts.append(int(t))
    off, mem = _csr(rows)
    return off, mem, np.array(ts, np.int64), int(mem.max()) + 1


def read_thyme_result(p: Path):
    """(runtime line, 96 counts) of a THyMe result file."""
    lines = p.read_text().split("\n")
    counts = np.zeros(96, np.uint64)
    for ln in lines[1:]:
        if ln.strip():
            i, c = ln.split("\t")
            counts[int(i) - 1] = int(c)
    return float(lines[0]), counts


def static_class_of_temporal() -> list[int]:
    """Static class (0..29) of each of the 96 temporal motifs: the motif's
    region pattern with the time order forgotten. Sums of the 96 counts over
    these groups do not depend on how ties in time are broken."""
    from oracle import oracle

    L = oracle.lib()
    pat = [0] * 96
    for p in range(128):
        m = L.hmo_temporal_class_bits(p)
        if m >= 0:
            pat[m] = p
    return [int(L.hmo_static_class_bits(p)) for p in pat]


def per_static(c96) -> list[int]:
    groups = static_class_of_temporal()
    out = [0] * 30
    for m in range(96):
        out[groups[m]] += int(c96[m])
    return out
