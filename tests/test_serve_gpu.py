"""Served requests over many resident graphs (hm_serve_*): every result is the
same in the batched mix, in the per-request form and on the graph alone, with
and without counts kept current by the exact deltas, and final counts match
the oracle."""
import numpy as np
import pytest

from tests.helpers import random_graph

pytestmark = pytest.mark.gpu


def _graphs(small=False):
    from ipdps26_b200 import gen

    ps = []
    sizes = [300, 1200, 60, 2500, 800, 40] if small else [3000, 12000, 600, 25000, 8000, 1500]
    for i, e in enumerate(sizes):
        q = 0.0 if e <= 3000 and i % 3 == 0 else 100.0  # plain-Zipf hubs on small graphs only
        ps.append(gen.params(500 + i, max(e // 2, 8), e, 2, 25, 2.5, 1.2, q))
    return ps, [gen.static(p) for p in ps]


def _trace(ps, n, seed, edits_max=800):
    from ipdps26_b200 import serve_trace

    return serve_trace.make_trace(ps, rate=1e6, duration=1e9, seed=seed, edits_min=5, edits_max=edits_max,
                                  max_requests=n)


def _run(ctx, hs, trace, mode, **kw):
    from ipdps26_b200 import engine, serve_trace

    with engine.Server(ctx, mode, **kw) as s:
        for h in hs:
            s.add_graph(h.offsets, h.members, h.n_nodes)
        s.start()
        rep = serve_trace.replay(s, trace, paced=False)
        live = [s.live_ids(k) for k in range(len(hs))]
        st = s.stats()
    return rep, live, st


def _alone(ctx, h, reqs):
    """The graph's own requests through the plain graph API."""
    from ipdps26_b200 import engine

    out = []
    with engine.Graph.from_hypergraph(ctx, h) as g:
        for r in reqs:
            if r.kind == engine.REQ_UPDATE:
                ids, d = g.apply_batch(r.dels, r.ins_off, r.ins_mem)
                out.append((ids, d, None))
            else:
                out.append((None, None, g.count_static30()))
    return out


@pytest.mark.parametrize("seed", [1, 2])
def test_batched_equals_per_request_equals_alone(ctx, seed):
    from ipdps26_b200 import engine, serve_trace

    ps, hs = _graphs(small=(seed == 1))
    trace = _trace(ps, 90, seed)
    rb, live_b, st_b = _run(ctx, hs, trace, engine.SERVE_BATCHED)
    rp, live_p, _ = _run(ctx, hs, trace, engine.SERVE_PER_REQUEST)
    assert all(r.status == 0 for r, _ in rb.results)
    assert serve_trace.same_results(rb, rp)
    assert all(np.array_equal(a, b) for a, b in zip(live_b, live_p))
    # submitted together, requests of different graphs shared rounds
    assert st_b.rounds < len(trace)
    assert max(r.round_requests for r, _ in rb.results) > 1
    # the ids the trace expects are the ids given
    for req, (r, ids) in zip(trace, rb.results):
        if req.kind == engine.REQ_UPDATE:
            assert np.array_equal(ids, req.ids)
    # each graph alone, through the plain API
    for k, h in enumerate(hs):
        mine = [(req, res) for req, res in zip(trace, rb.results) if req.graph == k]
        alone = _alone(ctx, h, [req for req, _ in mine])
        for (req, (r, ids)), (aids, ad, ac) in zip(mine, alone):
            if req.kind == engine.REQ_UPDATE:
                assert np.array_equal(ids, aids)
                assert list(r.delta30) == ad.tolist()
            else:
                assert list(r.counts30) == ac.tolist()


def test_final_counts_match_oracle(ctx):
    """After the whole trace, a count request of every graph equals the
    oracle's count of the graph's final hyperedges (rebuilt on the host)."""
    from ipdps26_b200 import engine, serve_trace
    from oracle import oracle

    ps, hs = _graphs(small=True)
    trace = _trace(ps, 60, 7, edits_max=200)
    final = [serve_trace.Request(1e9, k, engine.REQ_COUNT) for k in range(len(hs))]
    rep, _, _ = _run(ctx, hs, trace + final, engine.SERVE_BATCHED)
    rows = [{i: h.edge(i) for i in range(h.n_edges)} for h in hs]
    for req in trace:
        if req.kind != engine.REQ_UPDATE:
            continue
        e = rows[req.graph]
        for d in req.dels:
            del e[int(d)]
        for j, i in enumerate(req.ids):
            e[int(i)] = req.ins_mem[req.ins_off[j]:req.ins_off[j + 1]]
    for k, h in enumerate(hs):
        ids = sorted(rows[k])
        off = np.zeros(len(ids) + 1, np.uint64)
        off[1:] = np.cumsum([len(rows[k][i]) for i in ids])
        mem = np.concatenate([rows[k][i] for i in ids]).astype(np.uint32) if ids else np.zeros(0, np.uint32)
        r, _ = rep.results[len(trace) + k]
        assert list(r.counts30) == oracle.static30(off, mem, h.n_nodes).tolist(), k


def test_bad_requests_fail_alone(ctx):
    """A request that fails validation reports its status and changes
    nothing; the other requests of its round are served."""
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_INVALID, HM_ERR_NOT_LIVE

    ps, hs = _graphs(small=True)
    for mode in (engine.SERVE_BATCHED, engine.SERVE_PER_REQUEST):
        with engine.Server(ctx, mode) as s:
            for h in hs:
                s.add_graph(h.offsets, h.members, h.n_nodes)
            s.start()
            t_bad_id = s.submit_update(0, [hs[0].n_edges + 5])
            t_bad_node = s.submit_update(1, [], np.array([0, 2], np.uint64), np.array([0, hs[1].n_nodes], np.uint32))
            t_dup = s.submit_update(2, [1, 1])
            t_ok = s.submit_update(3, [0], np.array([0, 3], np.uint64), np.array([1, 2, 3], np.uint32))
            t_cnt = s.submit_count(0)
            s.drain()
            r1, _ = s.wait(t_bad_id)
            r2, _ = s.wait(t_bad_node)
            r3, _ = s.wait(t_dup)
            r4, ids4 = s.wait(t_ok)
            r5, _ = s.wait(t_cnt)
            assert r1.status == HM_ERR_NOT_LIVE
            assert r2.status == HM_ERR_INVALID
            assert r3.status == HM_ERR_INVALID
            assert r4.status == 0 and ids4.tolist() == [0]
            assert r5.status == 0
            assert len(s.live_ids(0)) == hs[0].n_edges
            assert len(s.live_ids(1)) == hs[1].n_edges
        with engine.Graph.from_hypergraph(ctx, hs[0]) as g:
            assert list(r5.counts30) == g.count_static30().tolist()


def test_budget_rejects_what_cannot_fit(ctx):
    """With an admission budget below the store itself, requests fail with
    HM_ERR_NOMEM before any device work, and the server stays usable."""
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_NOMEM

    ps, hs = _graphs(small=True)
    with engine.Server(ctx, engine.SERVE_BATCHED, mem_budget_bytes=1 << 20) as s:
        for h in hs:
            s.add_graph(h.offsets, h.members, h.n_nodes)
        s.start()
        t = s.submit_count(0)
        s.drain()
        r, _ = s.wait(t)
        assert r.status == HM_ERR_NOMEM


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_touch_orientations_agree_with_oracle(ctx, seed):
    """Touched-triple counts by (degree, id) rank and by id order agree, and
    equal count(G) - count(G without the marked hyperedges)."""
    from ipdps26_b200 import engine
    from oracle import oracle

    rng = np.random.default_rng(seed)
    off, mem = random_graph(rng, 300, 60, 10)
    n = len(off) - 1
    marked = np.sort(rng.choice(n, size=25, replace=False)).astype(np.uint32)
    keep = np.setdiff1d(np.arange(n), marked)
    rows = [mem[off[i]:off[i + 1]] for i in keep]
    off2 = np.zeros(len(rows) + 1, np.uint64)
    off2[1:] = np.cumsum([len(r) for r in rows])
    mem2 = np.concatenate(rows).astype(np.uint32)
    want = oracle.static30(off, mem, 60).astype(np.int64) - oracle.static30(off2, mem2, 60).astype(np.int64)
    with engine.Graph(ctx, off, mem, 60) as g:
        a = g.count_touching30(marked)
        g.set_touch_orientation(True)
        b = g.count_touching30(marked)
    assert a.astype(np.int64).tolist() == want.tolist()
    assert b.tolist() == a.tolist()


def test_id_orientation_deltas_match_recount(ctx):
    """Batches with the id-ordered walk give the same exact deltas."""
    from ipdps26_b200 import engine, gen

    p = gen.params(77, 2000, 4000, 2, 25, 2.5, 1.2, 0.0)
    h = gen.static(p)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        g.set_touch_orientation(True)
        total = g.count_static30().astype(np.int64)
        rng = np.random.default_rng(3)
        for b in range(4):
            dels, ins = gen.batch(p, 1000 + b, g.live_ids(), int(rng.integers(50, 600)))
            _, d = g.apply_batch(dels, ins.offsets, ins.members)
            total += d
            assert g.count_static30().astype(np.int64).tolist() == total.tolist()


@pytest.mark.parametrize("mode", ["batched", "per_request"])
def test_failed_round_is_reported_and_later_requests_fail_cleanly(ctx, mode):
    """Device allocation failure injected on the host in the middle of
    serving: the failing request reports HM_ERR_NOMEM, requests that depend
    on the damaged store report it too, none hangs, and the other graphs of
    the per-request form keep serving."""
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_NOMEM, lib

    ps, hs = _graphs(small=True)
    m = engine.SERVE_BATCHED if mode == "batched" else engine.SERVE_PER_REQUEST
    with engine.Server(ctx, m) as s:
        for h in hs:
            s.add_graph(h.offsets, h.members, h.n_nodes)
        s.start()
        ok, _ = s.wait(s.submit_update(0, [0], np.array([0, 2], np.uint64), np.array([1, 2], np.uint32)))
        assert ok.status == 0
        lib.hm_debug_fail_allocations_after(3)
        try:
            t1 = s.submit_update(1, [0, 1], np.array([0, 3], np.uint64), np.array([1, 2, 3], np.uint32))
            s.drain()
        finally:
            lib.hm_debug_fail_allocations_after(-1)
        r1, _ = s.wait(t1)
        assert r1.status == HM_ERR_NOMEM
        t2 = s.submit_update(1, [], np.array([0, 2], np.uint64), np.array([4, 5], np.uint32))
        t3 = s.submit_count(2)
        s.drain()
        r2, _ = s.wait(t2)
        r3, _ = s.wait(t3)
        assert r2.status == HM_ERR_NOMEM  # the damaged store refuses further work
        if mode == "batched":
            assert r3.status == HM_ERR_NOMEM  # one pooled store for all graphs
        else:
            assert r3.status == 0  # graph 2 has its own store
            with engine.Graph.from_hypergraph(ctx, hs[2]) as g:
                assert list(r3.counts30) == g.count_static30().tolist()


@pytest.mark.parametrize("seed", [1, 2])
def test_counts_from_deltas_equal_full_counts(ctx, seed):
    """count_from_deltas: counts kept current by the exact deltas answer the
    later count requests of each graph; every result equals the plain form,
    which counts in full every time."""
    from ipdps26_b200 import engine, serve_trace

    ps, hs = _graphs(small=(seed == 1))
    trace = _trace(ps, 90, seed)
    final = [serve_trace.Request(1e9, k, engine.REQ_COUNT) for k in range(len(hs))]
    full, live_f, _ = _run(ctx, hs, trace + final, engine.SERVE_PER_REQUEST)
    assert sum(r.kind == engine.REQ_COUNT for r in trace) > len(hs)  # graphs counted more than once
    for mode in (engine.SERVE_BATCHED, engine.SERVE_PER_REQUEST):
        kept, live_k, _ = _run(ctx, hs, trace + final, mode, count_from_deltas=True)
        assert all(r.status == 0 for r, _ in kept.results)
        assert serve_trace.same_results(full, kept), mode
        assert all(np.array_equal(a, b) for a, b in zip(live_f, live_k))


def test_counts_from_deltas_survive_rejected_updates(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_NOT_LIVE

    ps, hs = _graphs(small=True)
    off, mem = np.array([0, 3], np.uint64), np.array([1, 2, 3], np.uint32)
    for mode in (engine.SERVE_BATCHED, engine.SERVE_PER_REQUEST):
        with engine.Server(ctx, mode, count_from_deltas=True) as s:
            for h in hs:
                s.add_graph(h.offsets, h.members, h.n_nodes)
            s.start()
            r0, _ = s.wait(s.submit_count(0))
            bad, _ = s.wait(s.submit_update(0, [hs[0].n_edges + 5]))
            ok, _ = s.wait(s.submit_update(0, [0], off, mem))
            r1, _ = s.wait(s.submit_count(0))
        assert bad.status == HM_ERR_NOT_LIVE and ok.status == 0
        with engine.Graph.from_hypergraph(ctx, hs[0]) as g:
            assert list(r0.counts30) == g.count_static30().tolist()
            _, d = g.apply_batch([0], off, mem)
            assert list(ok.delta30) == d.tolist()
            assert list(r1.counts30) == g.count_static30().tolist()
