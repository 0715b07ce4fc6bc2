"""Keyed fill / unfill of live hyperedges (the reference's fillCBST /
CBSTOperations::insert(keys, payload, prefix) and unfillCBST) and the
stream-ordered variants of the batch update and the temporal count, on the
GPU, against a host mirror counted by the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle
from tests.helpers import csr

pytestmark = pytest.mark.gpu

HM_ERR_INVALID, HM_ERR_NOT_LIVE = -1, -5


def _oracle30(rows, n_nodes):
    off, mem = csr([rows[i] for i in sorted(rows)])
    return oracle.static30(off, mem, n_nodes).astype(np.int64)


@pytest.mark.parametrize("seed", range(3))
def test_keyed_fill_and_unfill_keep_ids_and_match_the_oracle(ctx, seed):
    from ipdps26_b200 import engine

    rng = np.random.default_rng(300 + seed)
    n_nodes = 50
    rows = [sorted(set(rng.choice(n_nodes, size=int(rng.integers(1, 7)), replace=False).tolist()))
            for _ in range(120)]
    mirror = dict(enumerate(rows))
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, n_nodes) as g:
        g.apply_batch([3, 9, 40])  # some free ids among the live ones
        for d in (3, 9, 40):
            del mirror[d]
        total = g.count_static30().astype(np.int64)
        assert total.tolist() == _oracle30(mirror, n_nodes).tolist()
        live_before = g.live_ids().tolist()
        for step in range(8):
            live = sorted(mirror)
            ids = rng.choice(live, size=int(rng.integers(1, 15)), replace=False).tolist()
            remove = step % 2 == 1
            vals = []
            for i in ids:
                have = mirror[i]
                if remove:
                    # some members, some non-members; every few steps all of them
                    k = len(have) if step % 4 == 3 else int(rng.integers(0, len(have) + 1))
                    v = list(rng.choice(have, size=k, replace=False)) if k else []
                    v += rng.integers(0, n_nodes, size=2).tolist()
                    mirror[i] = sorted(set(have) - set(v))
                else:
                    v = rng.integers(0, n_nodes, size=int(rng.integers(0, 5))).tolist() + have[:1]
                    mirror[i] = sorted(set(have) | set(v))
                vals.append(v)
            delta = g.unfill(ids, vals) if remove else g.fill(ids, vals)
            assert g.live_ids().tolist() == live_before, "ids are kept"
            for i, members in zip(ids, g.query(ids)):
                assert members.tolist() == mirror[i], (step, i)
            full = g.count_static30().astype(np.int64)
            assert full.tolist() == _oracle30(mirror, n_nodes).tolist(), step
            assert (total + delta).tolist() == full.tolist(), f"step {step}: delta"
            total = full
        # an emptied hyperedge comes back with a fill
        empty = [i for i in sorted(mirror) if not mirror[i]]
        if empty:
            delta = g.fill(empty[:1], [[0, 1, 2]])
            mirror[empty[0]] = [0, 1, 2]
            full = g.count_static30().astype(np.int64)
            assert full.tolist() == _oracle30(mirror, n_nodes).tolist()
            assert (total + delta).tolist() == full.tolist()


def test_fill_rejects_bad_calls_and_changes_nothing(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HmError

    rows = [[0, 1], [1, 2], [2, 3], [3, 0]]
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, 6) as g:
        g.apply_batch([2])
        before = g.count_static30().tolist()
        for ids, vals, status in (([2], [[4]], HM_ERR_NOT_LIVE), ([7], [[4]], HM_ERR_NOT_LIVE),
                                  ([0, 0], [[4], [5]], HM_ERR_INVALID), ([1], [[6]], HM_ERR_INVALID)):
            with pytest.raises(HmError) as e:
                g.fill(ids, vals)
            assert e.value.status == status, (ids, vals)
        assert g.count_static30().tolist() == before
        assert [m.tolist() for m in g.query([0, 1, 3])] == [[0, 1], [1, 2], [0, 3]]


def test_apply_batch_async_orders_on_the_callers_stream(ctx):
    """The batch starts after the caller's queued work and its delta lands
    in device memory before the caller's later work reads it; the ids and
    the delta equal those of the synchronous call on a twin graph."""
    import torch

    from ipdps26_b200 import engine, gen

    p = gen.config1(seed=31, n_nodes=500, n_edges=900)
    h = gen.static(p)
    with engine.Graph.from_hypergraph(ctx, h) as g, engine.Graph.from_hypergraph(ctx, h) as twin:
        s = torch.cuda.Stream(device=0)
        for b, where in enumerate(("side stream", "default stream", "context stream")):
            dels, ins = gen.batch(p, 500 + b, twin.live_ids(), 80)
            ids_sync, delta_sync = twin.apply_batch(dels, ins.offsets, ins.members)
            if where == "side stream":  # fill, update and read all queued on s
                with torch.cuda.stream(s):
                    out = torch.full((30,), 12345, dtype=torch.int64, device="cuda:0")
                ids = g.apply_batch_async(dels, ins.offsets, ins.members, out.data_ptr(), s.cuda_stream)
                with torch.cuda.stream(s):
                    got = out.cpu()
            elif where == "default stream":  # stream 0, torch's default stream
                out = torch.full((30,), 12345, dtype=torch.int64, device="cuda:0")
                ids = g.apply_batch_async(dels, ins.offsets, ins.members, out.data_ptr(), 0)
                got = out.cpu()
            else:  # the context stream is the engine's own: the caller synchronizes
                out = torch.full((30,), 12345, dtype=torch.int64, device="cuda:0")
                torch.cuda.synchronize()
                ids = g.apply_batch_async(dels, ins.offsets, ins.members, out.data_ptr(), None)
                torch.cuda.synchronize()
                got = out.cpu()
            assert ids.tolist() == ids_sync.tolist(), where
            assert got.numpy().tolist() == delta_sync.tolist(), where
        assert g.count_static30().tolist() == twin.count_static30().tolist()


def test_count_temporal_async_matches_the_synchronous_count(ctx):
    import torch

    from ipdps26_b200 import engine, gen

    t = gen.temporal(gen.params(7, 300, 1500, 2, 8, 2.5, 1.2, 0.0, dedupe=False), burst_rate=1e-3,
                     events_per_burst=20, gap_mean=5.0, span=200_000)
    with engine.Graph.from_hypergraph(ctx, t) as g:
        want = {d: g.count_temporal(d) for d in (500, 5000)}
        s = torch.cuda.Stream(device=0)
        for d in (500, 5000):
            with torch.cuda.stream(s):
                out = torch.full((96,), -1, dtype=torch.int64, device="cuda:0")
            g.count_temporal_async(d, out.data_ptr(), s.cuda_stream)
            with torch.cuda.stream(s):
                got = out.cpu().numpy().view(np.uint64)
            assert got.tolist() == want[d].tolist(), d
            out = torch.full((96,), -1, dtype=torch.int64, device="cuda:0")
            g.count_temporal_async(d, out.data_ptr(), 0)  # the legacy default stream
            assert out.cpu().numpy().view(np.uint64).tolist() == want[d].tolist(), d
        assert want[5000].tolist() == oracle.temporal96(t.offsets, t.members, t.timestamps, 5000).tolist()


def test_temporal_traffic_counts_the_window_projection(ctx):
    """hm_graph_temporal_traffic: sum of window degrees, adjacent pairs among
    each event's neighbours, and pairs (b, c) with c adjacent to a neighbour b
    but not to the event, against a direct enumeration on the host."""
    from ipdps26_b200 import engine, gen

    t = gen.temporal(gen.params(9, 60, 400, 2, 5, 2.5, 1.0, 0.0, dedupe=False), burst_rate=1e-3,
                     events_per_burst=15, gap_mean=4.0, span=40_000)
    delta = 300
    rows = [frozenset(t.edge(e).tolist()) for e in range(t.n_edges)]
    order = sorted(range(t.n_edges), key=lambda e: (int(t.timestamps[e]), e))
    first = {}
    sid = [first.setdefault(r, e) for e, r in enumerate(rows)]
    nb_sum = closed = open_b = 0
    for p, a in enumerate(order):
        ta = int(t.timestamps[a])
        window = {}  # static id -> node-set, events at most delta older, before a
        for q in order[:p]:
            if int(t.timestamps[q]) + delta >= ta and sid[q] != sid[a]:
                window.setdefault(sid[q], rows[q])
        nbrs = [x for x, r in window.items() if r & rows[a]]
        nb_sum += len(nbrs)
        ns = set(nbrs)
        for i, b in enumerate(nbrs):
            for c in nbrs[i + 1:]:
                closed += bool(window[b] & window[c])
            for c, r in window.items():
                if c != b and c not in ns and r & window[b]:
                    open_b += 1
    with engine.Graph.from_hypergraph(ctx, t) as g:
        g.count_temporal(delta)
        tr = g.temporal_traffic()
    assert (tr.window_neighbours, tr.closed_pairs, tr.open_pairs) == (nb_sum, closed, open_b)
    assert tr.b_temp == 8 * nb_sum + 8 * (nb_sum + 2 * closed + open_b)
