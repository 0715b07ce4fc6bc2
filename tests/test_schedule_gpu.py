"""Launch schedules of the static and touched-triple counts, the autotuner
that picks them, and the captured count graphs: counts are the reference's
under every schedule, before and after tuning, and when a captured count is
replayed or has to be captured again after an update; update deltas equal
recounts under every touched-triple schedule."""
import numpy as np
import pytest

from oracle import oracle
from tests.helpers import digest, load_golden, static_case

pytestmark = pytest.mark.gpu

# (warp_row, small_row): the default, every row in the large-table launch,
# no warp launch, no 4096-slot launch, and uneven splits
SCHEDULES = [(128, 2048), (0, 0), (0, 2048), (128, 128), (1, 64), (64, 1024), (17, 300)]
DEFAULT = (128, 2048, 128, 2048)


def _golden(name):
    rec = load_golden("static")[name]
    h = static_case(rec["params"])
    assert digest(h) == rec["sha256"]
    return h, rec["counts26"]


@pytest.mark.parametrize("name", ["c1law-2k-0", "c2law-3k", "wide-overlaps"])
def test_counts_equal_under_every_schedule(ctx, name):
    from ipdps26_b200 import engine

    h, want26 = _golden(name)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        assert g.schedule == DEFAULT
        base30 = g.count_static30()
        triads = g.count_vertex_triads()
        for s in SCHEDULES:
            g.set_schedule(*s)
            assert g.schedule == (*s, 128, 2048)
            assert g.count_static().tolist() == want26, s
            assert g.count_static30().tolist() == base30.tolist(), s
            assert g.count_vertex_triads().tolist() == triads.tolist(), s
            # partials add modulo 2^64 (a shard's open-pair classes may be negative)
            parts = sum(g.count_static30_shard(k, 3) for k in range(3))
            assert parts.tolist() == base30.tolist(), s


def test_schedule_rejects_what_the_kernels_cannot_hold(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_INVALID, HmError

    h, _ = _golden("wide-overlaps")
    with engine.Graph.from_hypergraph(ctx, h) as g:
        g.set_schedule(64, 512, 32, 1024)
        for bad in [(129, 2048), (64, 32), (0, 2049), (64, 512, 129, 2048), (64, 512, 64, 32), (64, 512, 0, 2049)]:
            with pytest.raises(HmError) as e:
                g.set_schedule(*bad)
            assert e.value.status == HM_ERR_INVALID
            assert g.schedule == (64, 512, 32, 1024)


@pytest.mark.parametrize("stride", [0, 1, 3])
def test_autotune_keeps_a_candidate_and_exact_counts(ctx, stride):
    from ipdps26_b200 import engine

    h, want26 = _golden("c1law-2k-1")
    with engine.Graph.from_hypergraph(ctx, h) as g:
        r = g.autotune(stride)
        d = r.as_dict()
        assert 1 < r.n_candidates <= engine.TUNE_MAX_CANDIDATES
        assert 1 < r.touch_n_candidates <= engine.TUNE_MAX_CANDIDATES
        assert d["static"]["default"] == [128, 2048] and d["touch"]["default"] == [128, 2048]
        assert r.best < r.n_candidates and r.touch_best < r.touch_n_candidates
        assert g.schedule == (*d["static"]["best"], *d["touch"]["best"])
        assert r.sample_stride == (stride or 1)  # 2000 hyperedges: one sample of all centres
        assert r.sampled > 0
        assert r.touch_sampled == h.n_edges  # fewer than 4096 live: every one marked
        assert all(r.ms[i] > 0 for i in range(r.n_candidates))
        assert all(r.touch_ms[i] > 0 for i in range(r.touch_n_candidates))
        # a default stays unless another candidate is at least 2 % faster
        if r.best:
            assert r.ms[r.best] <= 0.9801 * r.ms[0]
        if r.touch_best:
            assert r.touch_ms[r.touch_best] <= 0.9801 * r.touch_ms[0]
        assert g.count_static().tolist() == want26
        # deltas under the tuned touched-triple schedule
        before = g.count_static30().astype(np.int64)
        dels = np.arange(0, h.n_edges, 7, dtype=np.uint32)
        _, delta = g.apply_batch(dels)
        assert (before + delta).tolist() == g.count_static30().astype(np.int64).tolist()


def test_autotune_of_a_graph_without_triangles(ctx):
    from ipdps26_b200 import engine

    off = np.array([0, 2, 4], np.uint64)
    mem = np.array([0, 1, 2, 3], np.uint32)
    with engine.Graph(ctx, off, mem, 4) as g:
        r = g.autotune()
        assert r.sampled == 0 and r.best == 0 and r.touch_sampled == 2
        assert g.schedule[:2] == (128, 2048)
        assert int(g.count_static30().sum()) == 0


def test_captured_count_replays_and_recaptures_after_updates(ctx):
    """The second count of an unchanged graph replays the captured launches;
    updates and schedule changes make the next count capture again. Every
    count equals the oracle on a host mirror of the graph."""
    from ipdps26_b200 import engine, gen

    p = gen.params(31, 400, 800, 2, 25, 2.5, 1.2, 20.0)
    h = gen.static(p)
    rows = {i: h.edge(i) for i in range(h.n_edges)}

    def want():
        ids = sorted(rows)
        off = np.zeros(len(ids) + 1, np.uint64)
        off[1:] = np.cumsum([len(rows[i]) for i in ids])
        mem = np.concatenate([rows[i] for i in ids]).astype(np.uint32)
        return oracle.static30(off, mem, h.n_nodes).tolist()

    with engine.Graph.from_hypergraph(ctx, h) as g:
        first = g.count_static30().tolist()
        assert first == want()
        assert g.count_static30().tolist() == first  # replay
        for b in range(3):
            dels, ins = gen.batch(p, 500 + b, g.live_ids(), 120)
            ids, _ = g.apply_batch(dels, ins.offsets, ins.members)
            for d in dels:
                del rows[int(d)]
            for j, i in enumerate(ids):
                rows[int(i)] = ins.members[ins.offsets[j]:ins.offsets[j + 1]]
            w = want()
            assert g.count_static30().tolist() == w, b
            assert g.count_static30().tolist() == w, b  # replay
            g.set_schedule(*SCHEDULES[1 + b])
            assert g.count_static30().tolist() == w, b
        g.set_schedule(128, 2048)
        assert g.count_static30().tolist() == want()


def _without(h, marked):
    keep = np.setdiff1d(np.arange(h.n_edges), marked)
    rows = [h.edge(i) for i in keep]
    off = np.zeros(len(rows) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return off, np.concatenate(rows).astype(np.uint32)


@pytest.mark.parametrize("by_id", [False, True])
def test_touching_counts_equal_under_every_touch_schedule(ctx, by_id):
    """count_touching30(M) = count(G) - count(G without M) under every
    touched-triple split, in both walk orders."""
    from ipdps26_b200 import engine

    h, _ = _golden("c1law-2k-0")
    marked = np.sort(np.random.default_rng(5).choice(h.n_edges, size=300, replace=False)).astype(np.uint32)
    off2, mem2 = _without(h, marked)
    with engine.Graph(ctx, off2, mem2, h.n_nodes) as g2:
        rest = g2.count_static30()
    with engine.Graph.from_hypergraph(ctx, h) as g:
        g.set_touch_orientation(by_id)
        want = g.count_static30() - rest  # no class loses triples when hyperedges are added
        for t in SCHEDULES:
            g.set_schedule(128, 2048, *t)
            assert g.schedule == (128, 2048, *t)
            assert g.count_touching30(marked).tolist() == want.tolist(), t


def test_update_deltas_under_touch_schedules(ctx):
    from ipdps26_b200 import engine, gen

    p = gen.params(77, 2000, 4000, 2, 25, 2.5, 1.2, 0.0)
    h = gen.static(p)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        total = g.count_static30().astype(np.int64)
        for b, t in enumerate(SCHEDULES[1:5]):
            g.set_schedule(64, 1024, *t)
            dels, ins = gen.batch(p, 2000 + b, g.live_ids(), 400)
            _, d = g.apply_batch(dels, ins.offsets, ins.members)
            total += d
            assert g.count_static30().astype(np.int64).tolist() == total.tolist(), t
