"""The allocation-free touched-triple count, for callers that cannot call
cudaMalloc while they run (a serving loop that must not block on the
allocator, code held to a fixed memory reservation). It must give the same
30 counts as the allocating hm_count_touching30 and as the oracle
(count(G) - count(G without the marked hyperedges)), call after call, from
device buffers owned by the caller. This file is collected last so that a
failure here does not hide the other tests."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from tests.helpers import csr

pytestmark = pytest.mark.gpu

HM_ERR_NOT_LIVE = -5
HM_ERR_LIMIT = -8


def _call(g, ids_dev, n, out_dev, stream=None) -> int:
    """Raw status of hm_count_touching30_noalloc (stream: a cudaStream_t as
    an int, None for NULL, the legacy default stream)."""
    from ipdps26_b200._lib import lib

    fn = lib.hm_count_touching30_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    return fn(g.handle, C.c_void_p(ids_dev), n, C.c_void_p(out_dev), C.c_void_p(stream) if stream else None)


def _noalloc(g, ids_dev, n, out_dev, stream=None):
    from ipdps26_b200._lib import check

    check(_call(g, ids_dev, n, out_dev, stream), "hm_count_touching30_noalloc")


def _without(offsets, members, drop):
    """CSR of the hyperedges whose ids are not in `drop`."""
    drop = set(int(x) for x in drop)
    rows = [members[offsets[e]:offsets[e + 1]] for e in range(len(offsets) - 1) if e not in drop]
    return csr(rows)


def _oracle_touching(offsets, members, n_nodes, ids):
    full = oracle.static30(offsets, members, n_nodes).astype(np.int64)
    off2, mem2 = _without(offsets, members, ids)
    rest = oracle.static30(off2, mem2, n_nodes).astype(np.int64)
    return (full - rest).astype(np.uint64)


def _dev_ids(ids):
    import torch

    return torch.from_numpy(np.ascontiguousarray(ids, np.uint32).view(np.int32)).to("cuda:0")


def _host(out):
    return out.cpu().numpy().view(np.uint64)


def test_noalloc_matches_allocating_call_twice_in_a_row():
    import torch

    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=21, n_nodes=700, n_edges=1500))
    with engine.Context(0) as ctx, engine.Graph.from_hypergraph(ctx, h) as g:
        rng = np.random.default_rng(21)
        out = torch.zeros(30, dtype=torch.int64, device="cuda:0")
        for n in (40, 400):  # two calls in a row, on different id sets
            ids = np.unique(rng.choice(h.n_edges, size=n, replace=False)).astype(np.uint32)
            want = g.count_touching30(ids)
            ids_dev = _dev_ids(ids)
            out.fill_(-1)
            torch.cuda.synchronize()
            _noalloc(g, ids_dev.data_ptr(), len(ids), out.data_ptr())
            assert _host(out).tolist() == want.tolist(), n
        # the second set against the oracle directly
        assert want.tolist() == _oracle_touching(h.offsets, h.members, h.n_nodes, ids).tolist()


def _hub_graph(seed=7, per_node=20, hub_size=255):
    """One hub hyperedge of hub_size members, each member node shared with
    per_node other hyperedges of 2-4 members (so the hub has more than 4096
    neighbours and more than 64 members), plus a few hyperedges of 65-120
    members that overlap the hub and each other."""
    rng = np.random.default_rng(seed)
    n_extra = 3000
    hub = list(range(hub_size))
    rows = [hub]
    for v in hub:
        for _ in range(per_node):
            k = int(rng.integers(1, 4))
            rows.append([v] + list(hub_size + rng.choice(n_extra, size=k, replace=False)))
    for _ in range(6):
        k = int(rng.integers(65, 121))
        rows.append(list(rng.choice(hub_size + n_extra, size=k, replace=False)))
    off, mem = csr(rows)
    return off, mem, hub_size + n_extra


def test_noalloc_long_rows_and_large_hyperedges():
    """A marked hub whose row is longer than the kernel's shared-memory table
    (global binary search) and whose size is above 64 (triple overlaps by a
    three-way merge instead of position masks), together with marked
    hyperedges of 65-120 members; against the allocating call and the
    oracle."""
    import torch

    from ipdps26_b200 import engine

    off, mem, n_nodes = _hub_graph()
    n_edges = len(off) - 1
    with engine.Context(0) as ctx, engine.Graph(ctx, off, mem, n_nodes) as g:
        deg = g.info()
        assert deg.n_adjacent > 0
        ids = np.array([0, n_edges - 1, n_edges - 3, 17], np.uint32)  # hub, two large ones, one small
        want = _oracle_touching(off, mem, n_nodes, ids)
        assert g.count_touching30(ids).tolist() == want.tolist()
        out = torch.full((30,), -1, dtype=torch.int64, device="cuda:0")
        ids_dev = _dev_ids(ids)
        torch.cuda.synchronize()
        _noalloc(g, ids_dev.data_ptr(), len(ids), out.data_ptr())
        assert _host(out).tolist() == want.tolist()
        # only the hub: its row alone goes through the global search
        hub_dev = _dev_ids(np.array([0], np.uint32))
        want_hub = _oracle_touching(off, mem, n_nodes, [0])
        torch.cuda.synchronize()
        _noalloc(g, hub_dev.data_ptr(), 1, out.data_ptr())
        assert _host(out).tolist() == want_hub.tolist()


def test_noalloc_repeated_dead_and_out_of_range_ids():
    """Repeats count once; ids that are free or beyond the slots make the
    call return HM_ERR_NOT_LIVE while the live ids are still counted."""
    import torch

    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=23, n_nodes=500, n_edges=900))
    with engine.Context(0) as ctx, engine.Graph.from_hypergraph(ctx, h) as g:
        dead = np.array([5, 77, 300], np.uint32)
        g.apply_batch(dead)  # frees three ids
        live = np.array([3, 10, 11, 500, 640], np.uint32)
        want = g.count_touching30(live)
        off2, mem2 = _without(h.offsets, h.members, dead)
        # the oracle on the graph after the deletions (ids renumbered, counts unchanged)
        keep = np.setdiff1d(np.arange(h.n_edges, dtype=np.uint32), dead)
        renum = np.searchsorted(keep, live).astype(np.uint32)
        assert want.tolist() == _oracle_touching(off2, mem2, h.n_nodes, renum).tolist()
        info = g.info()
        ids = np.concatenate([live, live[:3], dead[:2], [info.n_slots + 5, 0xFFFFFFFF]]).astype(np.uint32)
        out = torch.full((30,), -1, dtype=torch.int64, device="cuda:0")
        ids_dev = _dev_ids(ids)
        torch.cuda.synchronize()
        assert _call(g, ids_dev.data_ptr(), len(ids), out.data_ptr()) == HM_ERR_NOT_LIVE
        assert _host(out).tolist() == want.tolist()
        # and a clean call right after it gives the same counts with HM_OK
        ids_dev = _dev_ids(live)
        out.fill_(-1)
        torch.cuda.synchronize()
        _noalloc(g, ids_dev.data_ptr(), len(live), out.data_ptr())
        assert _host(out).tolist() == want.tolist()


def test_noalloc_on_caller_streams():
    """On a torch side stream and on the legacy default stream (NULL): the
    caller's earlier work on that stream (the id upload, clearing the output)
    is ordered before the count, with no synchronize in between."""
    import torch

    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=25, n_nodes=600, n_edges=1100))
    with engine.Context(0) as ctx, engine.Graph.from_hypergraph(ctx, h) as g:
        ids = np.arange(0, h.n_edges, 7, dtype=np.uint32)
        want = g.count_touching30(ids)
        s = torch.cuda.Stream(device=0)
        with torch.cuda.stream(s):
            ids_dev = _dev_ids(ids)
            out = torch.full((30,), -1, dtype=torch.int64, device="cuda:0")
        _noalloc(g, ids_dev.data_ptr(), len(ids), out.data_ptr(), s.cuda_stream)
        with torch.cuda.stream(s):
            got = _host(out)
        assert got.tolist() == want.tolist()
        # the default stream: the fill below is queued, not waited for
        ids_dev = _dev_ids(ids)
        out = torch.full((30,), -1, dtype=torch.int64, device="cuda:0")
        _noalloc(g, ids_dev.data_ptr(), len(ids), out.data_ptr(), None)
        assert _host(out).tolist() == want.tolist()


def test_noalloc_rejects_sizes_beyond_its_limits():
    """More than 2^21 hyperedge slots, or more than 2^20 ids in one call:
    HM_ERR_LIMIT before any device work."""
    import torch

    from ipdps26_b200 import engine

    n = (1 << 21) + 1
    off = np.arange(n + 1, dtype=np.uint64)
    mem = np.arange(n, dtype=np.uint32)  # singletons: no adjacency
    out = torch.zeros(30, dtype=torch.int64, device="cuda:0")
    ids_dev = _dev_ids(np.zeros(4, np.uint32))
    with engine.Context(0) as ctx:
        with engine.Graph(ctx, off, mem, n) as g:
            assert _call(g, ids_dev.data_ptr(), 1, out.data_ptr()) == HM_ERR_LIMIT
        h_off, h_mem = csr([[0, 1], [1, 2], [2, 0]])
        with engine.Graph(ctx, h_off, h_mem, 3) as g:
            # the count is rejected on its size alone; the buffer is never read
            assert _call(g, ids_dev.data_ptr(), (1 << 20) + 1, out.data_ptr()) == HM_ERR_LIMIT
            _noalloc(g, ids_dev.data_ptr(), 1, out.data_ptr())
            assert _host(out).tolist() == g.count_touching30([0]).tolist()
