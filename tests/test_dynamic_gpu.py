"""Batch updates and the exact incremental recount on the GPU, against a host
mirror of the live hyperedges counted by the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle
from tests.helpers import csr

pytestmark = pytest.mark.gpu


class Mirror:
    """Host copy of the live hyperedges by id, with the engine's id rule."""

    def __init__(self, rows):
        self.rows = {i: sorted(set(r)) for i, r in enumerate(rows)}
        self.n_slots = len(rows)

    def apply(self, dels, ins_rows):
        for d in dels:
            del self.rows[d]
        free = sorted(set(range(self.n_slots)) - set(self.rows))
        ids = []
        for k, r in enumerate(ins_rows):
            if k < len(free):
                i = free[k]
            else:
                i = self.n_slots
                self.n_slots += 1
            self.rows[i] = sorted(set(r))
            ids.append(i)
        return ids

    def counts(self, n_nodes):
        live = [self.rows[i] for i in sorted(self.rows)]
        off, mem = csr(live)
        return oracle.static30(off, mem, n_nodes)


def random_rows(rng, n, n_nodes, kmax):
    return [list(rng.choice(n_nodes, size=int(rng.integers(1, kmax + 1)), replace=False)) for _ in range(n)]


@pytest.mark.parametrize("seed", range(4))
def test_batches_match_full_recount(ctx, seed):
    from ipdps26_b200 import engine

    rng = np.random.default_rng(seed)
    n_nodes = 60
    rows = random_rows(rng, 150, n_nodes, 6)
    mirror = Mirror(rows)
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, n_nodes) as g:
        total = g.count_static30().astype(np.int64)
        assert total.tolist() == mirror.counts(n_nodes).astype(np.int64).tolist()
        for step in range(6):
            live = np.array(sorted(mirror.rows), dtype=np.uint32)
            n_del = int(rng.integers(0, 25))
            dels = sorted(rng.choice(live, size=min(n_del, len(live)), replace=False).tolist())
            ins_rows = random_rows(rng, int(rng.integers(0, 30)), n_nodes, 6)
            want_ids = mirror.apply(dels, ins_rows)
            io, im = csr(ins_rows)
            ids, delta = g.apply_batch(dels, io, im)
            assert ids.tolist() == want_ids
            full = g.count_static30().astype(np.int64)
            want = mirror.counts(n_nodes).astype(np.int64)
            assert full.tolist() == want.tolist(), f"step {step}"
            assert (total + delta).tolist() == full.tolist(), f"step {step}: delta"
            total = full
            assert g.live_ids().tolist() == sorted(mirror.rows)
            q = g.query(ids[:5]) if len(ids) else []
            for i, members in zip(ids[:5], q):
                assert members.tolist() == mirror.rows[int(i)]


def test_delete_everything_then_reinsert(ctx):
    from ipdps26_b200 import engine

    rows = [[0, 1], [1, 2], [2, 0], [0, 3]]
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, 4) as g:
        before = g.count_static30()
        ids, delta = g.apply_batch([0, 1, 2, 3])
        assert (before.astype(np.int64) + delta).tolist() == [0] * 30
        assert g.count_static30().tolist() == [0] * 30
        io, im = csr(rows)
        ids, delta = g.apply_batch([], io, im)
        assert ids.tolist() == [0, 1, 2, 3]
        assert g.count_static30().tolist() == before.tolist()
        assert delta.tolist() == before.astype(np.int64).tolist()


def test_bad_batches_are_rejected(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HmError

    off, mem = csr([[0, 1], [1, 2]])
    with engine.Graph(ctx, off, mem, 3) as g:
        with pytest.raises(HmError) as e:
            g.apply_batch([5])
        assert e.value.status == -5
        with pytest.raises(HmError) as e:
            g.apply_batch([0, 0])
        assert e.value.status == -1
        io, im = csr([[0, 7]])
        with pytest.raises(HmError) as e:
            g.apply_batch([], io, im)
        assert e.value.status == -1
        assert g.count_static30().tolist() == oracle.static30(off, mem, 3).tolist()


def test_touching_counts(ctx):
    """Counts of triples touching a set = full count minus count without it."""
    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=4, n_nodes=200, n_edges=300))
    full = oracle.static30(h.offsets, h.members, h.n_nodes).astype(np.int64)
    marked = [3, 50, 51, 120, 299]
    rest = [h.edge(e).tolist() for e in range(h.n_edges) if e not in marked]
    off, mem = csr(rest)
    without = oracle.static30(off, mem, h.n_nodes).astype(np.int64)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        got = g.count_touching30(marked).astype(np.int64)
    assert got.tolist() == (full - without).tolist()


def test_c3_style_batches_on_config2_laws(ctx):
    """Log-uniform batch sizes, 80 % inserts / 20 % deletes, on a config-2-law
    graph; incremental == full recount after every batch."""
    from ipdps26_b200 import engine, gen

    p = gen.config2(seed=2, n_nodes=4000, n_edges=6000, q=3.0)
    h = gen.static(p)
    rng = np.random.default_rng(2)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        total = g.count_static30().astype(np.int64)
        for b in range(5):
            n_edits = int(np.exp(rng.uniform(np.log(10), np.log(1000))))
            live = g.live_ids()
            dels, ins = gen.batch(p, 1000 + b, live, n_edits, 0.8)
            _, delta = g.apply_batch(dels, ins.offsets, ins.members)
            total = total + delta
            full = g.count_static30().astype(np.int64)
            assert total.tolist() == full.tolist()
