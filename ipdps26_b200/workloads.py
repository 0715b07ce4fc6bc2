"""Parameters of the named synthetic workloads, as plain data.

Nothing here loads the engine: a process that times the reference's own
counters reads these and writes the inputs with the host-only ``hmgen`` tool
(``ipdps26_b200/hmgen``, built from the generator sources without CUDA), so it
counts exactly the hyperedges the engine counts without mapping the engine.
``gen`` turns the same parameters into generator calls.

Popularity is Zipf-Mandelbrot, P(rank r) ~ (r + 1 + q)^-s, q the offset.
"""
from __future__ import annotations

import subprocess
from dataclasses import asdict, dataclass, replace
from pathlib import Path

HMGEN = Path(__file__).resolve().parent / "hmgen"


@dataclass(frozen=True)
class Laws:
    seed: int
    n_nodes: int
    n_edges: int
    k_min: int
    k_max: int
    size_exp: float
    pop_exp: float
    q: float = 0.0
    dedupe: bool = True

    def scaled(self, **kw) -> "Laws":
        return replace(self, **kw)

    def as_dict(self) -> dict:
        return asdict(self)


@dataclass(frozen=True)
class Bursts:
    burst_rate: float = 1e-4
    events_per_burst: int = 50
    gap_mean: float = 20.0
    span: int = 100_000_000


# Config 1: 10K nodes, 20K hyperedges, sizes k^-2.5 on [2,25], Zipf(1.2).
CONFIG1 = Laws(0, 10_000, 20_000, 2, 25, 2.5, 1.2, 0.0)

# Config 2: 1M nodes, 2M hyperedges, sizes k^-2.2 on [2,100], Zipf-Mandelbrot
# s = 1.1 with offset q = 1000 (plain Zipf(1.1) makes the projection of this
# size exceed device memory and any exact counter: a hub of degree ~770K and
# about 1.1e17 triples sharing one node).
C2_Q = 1000.0
CONFIG2 = Laws(1, 1_000_000, 2_000_000, 2, 100, 2.2, 1.1, C2_Q)

# Config 4: 500K timestamped hyperedges over 200K nodes, sizes k^-2.5 on
# [2,20], Zipf(1.2); repeated node-sets are kept (they make motifs 87-96);
# bursty times over a span of 1e8, made strictly increasing.
CONFIG4 = Laws(3, 200_000, 500_000, 2, 20, 2.5, 1.2, 0.0, dedupe=False)
CONFIG4_BURSTS = Bursts()

# Config 5 graphs use the config-1 laws with q = 1000 (see gen.config5_graph).
C5_Q = 1000.0


def config2_laws(n_edges: int = CONFIG2.n_edges, n_nodes: int = CONFIG2.n_nodes) -> Laws:
    """Config 2's laws at another size; q scales with the number of
    hyperedges so that the hub degree keeps its share."""
    return CONFIG2.scaled(n_edges=n_edges, n_nodes=n_nodes, q=C2_Q * n_edges / CONFIG2.n_edges)


def write_static(laws: Laws, path, prefix: int = 0, fmt: str = "mochy") -> tuple[int, int]:
    """Writes the workload (its first `prefix` hyperedges when prefix > 0) in
    MoCHy's (or ESCHER's) text format with hmgen; returns (hyperedges, nodes)."""
    L = laws
    cmd = [str(HMGEN), "static", str(L.seed), str(L.n_nodes), str(L.n_edges), str(L.k_min), str(L.k_max),
           repr(L.size_exp), repr(L.pop_exp), repr(L.q), str(int(L.dedupe)), str(prefix), str(path), fmt]
    r = subprocess.run(cmd, capture_output=True, text=True, check=True)
    e, n = r.stdout.split()
    return int(e), int(n)


def write_temporal(laws: Laws, bursts: Bursts, path, prefix: int = 0) -> tuple[int, int]:
    """Writes the temporal workload (or its first `prefix` events) as THyMe
    input ("nodes<TAB>time" lines) with hmgen; returns (events, nodes)."""
    L, B = laws, bursts
    cmd = [str(HMGEN), "temporal", str(L.seed), str(L.n_nodes), str(L.n_edges), str(L.k_min), str(L.k_max),
           repr(L.size_exp), repr(L.pop_exp), repr(L.q), str(int(L.dedupe)), repr(B.burst_rate),
           str(B.events_per_burst), repr(B.gap_mean), str(B.span), str(prefix), str(path)]
    r = subprocess.run(cmd, capture_output=True, text=True, check=True)
    e, n = r.stdout.split()
    return int(e), int(n)
