"""Host side of the served workload, without a GPU: the id rule the traces
follow (the one hm_graph_apply_batch and the server use), seeded traces whose
deletions always name live hyperedges, and the summaries and comparisons the
serving tests and the bench rely on."""
import numpy as np

from ipdps26_b200 import engine, gen, serve_trace


def test_id_mirror_smallest_free_first():
    m = serve_trace.IdMirror(6)
    # freed ids are reused ascending (those freed by the same batch included), then new ids
    assert m.apply(np.array([4, 1], np.uint32), 3).tolist() == [1, 4, 6]
    assert m.live_ids().tolist() == [0, 1, 2, 3, 4, 5, 6]
    assert m.apply(np.array([0, 6, 2], np.uint32), 1).tolist() == [0]
    assert m.live_ids().tolist() == [0, 1, 3, 4, 5]
    assert m.apply(np.zeros(0, np.uint32), 3).tolist() == [2, 6, 7]
    assert m.apply(np.array([7], np.uint32), 0).tolist() == []
    assert m.live_ids().tolist() == [0, 1, 2, 3, 4, 5, 6]


def _graphs():
    return [gen.params(300 + i, 100, 200 + 50 * i, 2, 8, 2.5, 1.2, 10.0) for i in range(4)]


def test_trace_is_seeded():
    ps = _graphs()
    a = serve_trace.make_trace(ps, rate=1e4, duration=0.01, seed=3, edits_min=5, edits_max=50)
    b = serve_trace.make_trace(ps, rate=1e4, duration=0.01, seed=3, edits_min=5, edits_max=50)
    c = serve_trace.make_trace(ps, rate=1e4, duration=0.01, seed=4, edits_min=5, edits_max=50)
    assert len(a) > 20 and len(a) == len(b)
    for x, y in zip(a, b):
        assert (x.t, x.graph, x.kind) == (y.t, y.graph, y.kind)
        for f in ("dels", "ins_off", "ins_mem", "ids"):
            assert np.array_equal(getattr(x, f), getattr(y, f))
    assert [(x.graph, x.kind) for x in a] != [(x.graph, x.kind) for x in c]


def test_trace_deletions_name_live_hyperedges_in_arrival_order():
    """Served in arrival order, every deletion names a live id of its graph,
    and the ids the trace expects for the insertions are the rule's."""
    ps = _graphs()
    trace = serve_trace.make_trace(ps, rate=1e4, duration=0.02, seed=9, edits_min=5, edits_max=80)
    live = [set(range(p.n_edges)) for p in ps]
    kinds = {engine.REQ_UPDATE: 0, engine.REQ_COUNT: 0}
    last_t = 0.0
    for r in trace:
        assert r.t >= last_t
        last_t = r.t
        kinds[r.kind] += 1
        if r.kind != engine.REQ_UPDATE:
            continue
        s = live[r.graph]
        assert len(set(r.dels.tolist())) == len(r.dels)
        assert all(int(d) in s for d in r.dels)
        s.difference_update(int(d) for d in r.dels)
        n_ins = len(r.ins_off) - 1
        assert r.edits == len(r.dels) + n_ins
        want, cand = [], 0
        while len(want) < n_ins:
            if cand not in s:
                want.append(cand)
            cand += 1
        assert r.ids.tolist() == want
        s.update(want)
        # inserted members are sorted, distinct and inside the graph's node range
        for j in range(n_ins):
            row = r.ins_mem[r.ins_off[j]:r.ins_off[j + 1]]
            assert len(row) >= 2 and np.all(np.diff(row.astype(np.int64)) > 0)
            assert int(row.max()) < ps[r.graph].n_nodes
    assert kinds[engine.REQ_UPDATE] > kinds[engine.REQ_COUNT] > 0


def _result(kind, status=0, delta=None, counts=None, submit=0.0, done=1.0, rounds=1):
    r = engine.ServeResult()
    r.kind, r.status, r.submit_ms, r.done_ms, r.round_requests = kind, status, submit, done, rounds
    for k, v in enumerate(delta or []):
        r.delta30[k] = v
    for k, v in enumerate(counts or []):
        r.counts30[k] = v
    return r


def test_same_results_compares_every_field_it_promises():
    u = lambda d: (_result(engine.REQ_UPDATE, delta=d), np.array([3, 4], np.uint32))  # noqa: E731
    c = lambda n: (_result(engine.REQ_COUNT, counts=n), np.zeros(0, np.uint32))  # noqa: E731
    a = serve_trace.Replay([u([1, -2]), c([5, 6])], 1.0, 0.0)
    assert serve_trace.same_results(a, serve_trace.Replay([u([1, -2]), c([5, 6])], 2.0, 3.0))
    assert not serve_trace.same_results(a, serve_trace.Replay([u([1, -3]), c([5, 6])], 1.0, 0.0))
    assert not serve_trace.same_results(a, serve_trace.Replay([u([1, -2]), c([5, 7])], 1.0, 0.0))
    assert not serve_trace.same_results(a, serve_trace.Replay([u([1, -2])], 1.0, 0.0))
    other_ids = (_result(engine.REQ_UPDATE, delta=[1, -2]), np.array([3, 5], np.uint32))
    assert not serve_trace.same_results(a, serve_trace.Replay([other_ids, c([5, 6])], 1.0, 0.0))
    failed = (_result(engine.REQ_UPDATE, status=-3, delta=[1, -2]), np.array([3, 4], np.uint32))
    assert not serve_trace.same_results(a, serve_trace.Replay([failed, c([5, 6])], 1.0, 0.0))


def test_summarize_throughput_and_latency():
    trace = [serve_trace.Request(0.0, 0, engine.REQ_UPDATE, np.array([1], np.uint32), np.array([0, 2], np.uint64),
                                 np.array([0, 1], np.uint32)),
             serve_trace.Request(0.1, 1, engine.REQ_COUNT)]
    res = [(_result(engine.REQ_UPDATE, submit=0.0, done=400.0, rounds=2), np.zeros(1, np.uint32)),
           (_result(engine.REQ_COUNT, submit=100.0, done=500.0, rounds=2), np.zeros(0, np.uint32))]
    sm = serve_trace.summarize(trace, serve_trace.Replay(res, 0.5, 0.0))
    assert sm["requests"] == 2 and sm["updates"] == 1 and sm["counts"] == 1 and sm["failed"] == 0
    assert sm["span_s"] == 0.5
    assert sm["update_batches_per_s"] == 2.0
    assert sm["edits_per_s"] == 4.0  # one deletion + one insertion in 0.5 s
    assert sm["update_p50_ms"] == 400.0 and sm["count_p50_ms"] == 400.0
    assert sm["mean_round_requests"] == 2.0
