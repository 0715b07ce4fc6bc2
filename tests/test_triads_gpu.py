"""Vertex-triad counts (the reference's type 1/2/3 programs) on the GPU
against the oracle, which is pinned to the reference's own counters."""
import numpy as np
import pytest

from tests.helpers import random_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_graphs(ctx, seed):
    from ipdps26_b200 import engine
    from oracle import oracle

    rng = np.random.default_rng(seed)
    off, mem = random_graph(rng, 300, 60, 12, p_repeat=0.1)
    with engine.Graph(ctx, off, mem, 60) as g:
        got = g.count_vertex_triads()
    assert got.tolist() == oracle.vertex_triads(off, mem).tolist()


def test_law_graph_with_large_hyperedges_and_updates(ctx):
    """Hub-heavy graph with hyperedges above 64 members (the merge path),
    recounted after an update batch."""
    from ipdps26_b200 import engine, gen
    from oracle import oracle

    p = gen.params(8, 200, 500, 2, 90, 1.8, 1.2, 0.0)
    h = gen.static(p)
    assert np.diff(h.offsets).max() > 64
    with engine.Graph.from_hypergraph(ctx, h) as g:
        assert g.count_vertex_triads().tolist() == oracle.vertex_triads(h.offsets, h.members).tolist()
        dels, ins = gen.batch(p, 99, g.live_ids(), 80)
        g.apply_batch(dels, ins.offsets, ins.members, delta=False)
        ids = g.live_ids()
        rows = g.query(ids)
        off = np.zeros(len(rows) + 1, np.uint64)
        off[1:] = np.cumsum([len(r) for r in rows])
        mem = np.concatenate(rows).astype(np.uint32)
        assert g.count_vertex_triads().tolist() == oracle.vertex_triads(off, mem).tolist()
