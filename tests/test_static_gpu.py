"""Static 26/30-class counts on the GPU, through the C ABI, against the
reference's outputs (golden fixtures) and the CPU oracle."""
from math import comb

import numpy as np
import pytest

from oracle import oracle, refdata
from tests.helpers import csr, digest, load_golden, random_graph, static_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(k for k in load_golden("static") if k != "dblp"))
def test_static_matches_mochy_golden(ctx, name):
    from ipdps26_b200 import engine

    rec = load_golden("static")[name]
    h = static_case(rec["params"])
    assert digest(h) == rec["sha256"]
    with engine.Graph.from_hypergraph(ctx, h) as g:
        assert g.count_static().tolist() == rec["counts26"]


def test_static_on_mochy_dblp(ctx):
    """MoCHy's own sample hypergraph (dblp_graph.txt) against the counts
    MoCHy main_exact printed for it."""
    from ipdps26_b200 import engine

    rec = load_golden("static")["dblp"]
    p = refdata.path("dblp")
    if p is None:
        pytest.skip("reference dataset not present (oracle/build_ref.sh copies it)")
    assert refdata.sha256(p) == rec["file_sha256"]
    off, mem, n_nodes = refdata.read_mochy(p)
    with engine.Graph(ctx, off, mem, n_nodes) as g:
        assert g.count_static().tolist() == rec["counts26"]


@pytest.mark.parametrize("seed", range(8))
def test_static_matches_oracle_random(ctx, seed):
    from ipdps26_b200 import engine

    rng = np.random.default_rng(seed)
    n_nodes = int(rng.integers(5, 80))
    off, mem = random_graph(rng, int(rng.integers(1, 300)), n_nodes, int(rng.integers(1, 12)), p_repeat=0.2)
    want = oracle.static30(off, mem, n_nodes)
    with engine.Graph(ctx, off, mem, n_nodes) as g:
        assert g.count_static30().tolist() == want.tolist()


def test_static_repeated_hyperedges(ctx):
    """Repeated hyperedges feed the four classes MoCHy does not report."""
    from ipdps26_b200 import engine

    rows = [[0, 1], [0, 1], [1, 2], [0, 1, 2], [0, 1, 2], [2, 3], [3], [3]]
    off, mem = csr(rows)
    want = oracle.static30(off, mem, 4)
    assert any(want[k] for k in (0, 1, 4, 6))
    with engine.Graph(ctx, off, mem, 4) as g:
        assert g.count_static30().tolist() == want.tolist()


@pytest.mark.parametrize("rows,n_nodes", [([], 1), ([[0]], 1), ([[0, 1]], 2), ([[0, 1], [2, 3]], 4),
                                         ([[0, 1], [1, 2]], 3)])
def test_static_tiny_edge_cases(ctx, rows, n_nodes):
    from ipdps26_b200 import engine

    off, mem = csr(rows)
    want = oracle.static30(off, mem, n_nodes)
    with engine.Graph(ctx, off, mem, n_nodes) as g:
        assert g.count_static30().tolist() == want.tolist()


@pytest.mark.parametrize("n", [300, 5000])
def test_static_star_clique(ctx, n):
    """n hyperedges {0, i}: every triple is closed with g = 1 (class 3).
    n = 5000 gives oriented rows longer than the shared-memory hash table."""
    from ipdps26_b200 import engine

    rows = [[0, i + 1] for i in range(n)]
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, n + 1) as g:
        got = g.count_static30()
    want = np.zeros(30, np.uint64)
    want[3] = comb(n, 3)
    assert got.tolist() == want.tolist()


def test_static_c1law_against_oracle(ctx):
    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=77, n_nodes=600, n_edges=1200))
    want = oracle.static30(h.offsets, h.members, h.n_nodes)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        assert g.count_static30().tolist() == want.tolist()
        assert g.count_static30().tolist() == want.tolist()  # repeatable


def test_query_returns_sorted_members(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HmError

    rows = [[5, 3, 3, 1], [2], [4, 0, 2]]
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, 6) as g:
        q = g.query([2, 0, 1])
        assert [x.tolist() for x in q] == [[0, 2, 4], [1, 3, 5], [2]]
        with pytest.raises(HmError) as e:
            g.query([3])
        assert e.value.status == -5


def test_build_rejects_bad_input(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HmError

    off, mem = csr([[0, 1], [1, 9]])
    with pytest.raises(HmError) as e:
        engine.Graph(ctx, off, mem, 5)
    assert e.value.status == -1
    off, mem = csr([list(range(300))])
    with pytest.raises(HmError) as e:
        engine.Graph(ctx, off, mem, 300)
    assert e.value.status == -8


@pytest.mark.parametrize("n_shards", [2, 3, 8])
def test_static_shards_sum_to_full_count(ctx, n_shards):
    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config2(seed=9, n_nodes=3000, n_edges=6000, q=3.0))
    with engine.Graph.from_hypergraph(ctx, h) as g:
        full = g.count_static30()
        parts = sum(g.count_static30_shard(s, n_shards) for s in range(n_shards))
    assert parts.tolist() == full.tolist()


def test_async_count_on_caller_and_context_streams(ctx):
    """hm_count_static30_async: queued after a caller's stream (twice in a
    row, reusing the graph's counters) and on the context stream, the counts
    reach the caller's device buffers and equal the oracle."""
    import torch

    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=78, n_nodes=600, n_edges=1200))
    want = oracle.static30(h.offsets, h.members, h.n_nodes)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        s = torch.cuda.Stream(device=0)
        outs = [torch.full((30,), -1, dtype=torch.int64, device="cuda:0") for _ in range(3)]
        torch.cuda.synchronize()
        g.count_static30_async(outs[0].data_ptr(), s.cuda_stream)
        g.count_static30_async(outs[1].data_ptr(), s.cuda_stream)
        s.synchronize()
        g.count_static30_async(outs[2].data_ptr(), None)
        torch.cuda.synchronize()
        for o in outs:
            assert o.cpu().numpy().view(np.uint64).tolist() == want.tolist()
        assert g.count_static30().tolist() == want.tolist()


def test_async_count_on_the_default_stream_without_synchronize(ctx):
    """Stream 0 (the legacy default stream, torch's default stream) is a
    caller's stream like any other: a fill queued on it before the count, and
    the read queued after it, are ordered with no explicit synchronize. The
    phase times of an asynchronous count read as not measured."""
    import torch

    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=79, n_nodes=700, n_edges=1400))
    want = oracle.static30(h.offsets, h.members, h.n_nodes)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        g.count_static30()  # prepared; later counts replay the captured launches
        for _ in range(3):
            out = torch.empty(30, dtype=torch.int64, device="cuda:0")
            out.fill_(-1)
            g.count_static30_async(out.data_ptr(), 0)
            assert out.cpu().numpy().view(np.uint64).tolist() == want.tolist()
        assert g.timings().closed_ms == -1.0


def test_async_count_refuses_a_capturing_stream(ctx):
    """A caller's stream under CUDA-graph capture is refused with
    HM_ERR_STATE; the capture itself stays usable."""
    import torch

    from ipdps26_b200 import engine, gen
    from ipdps26_b200._lib import HmError

    h = gen.static(gen.config1(seed=80, n_nodes=300, n_edges=500))
    with engine.Graph.from_hypergraph(ctx, h) as g:
        g.count_static30()
        out = torch.zeros(30, dtype=torch.int64, device="cuda:0")
        s = torch.cuda.Stream(device=0)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with pytest.raises(HmError) as ei:
                with torch.cuda.graph(graph, stream=s):
                    out.add_(1)
                    try:
                        g.count_static30_async(out.data_ptr(), s.cuda_stream)
                    finally:
                        out.add_(1)
        assert ei.value.status == -7
        torch.cuda.synchronize()
        assert g.count_static30().tolist() == oracle.static30(h.offsets, h.members, h.n_nodes).tolist()


def _heavy_rich_rows(rng):
    """Hyperedges built so that the static count's grouped walk meets every
    case: hubs 0 and 1 shared by 300 hyperedges (each pair shares both, so
    centres have far more heavy neighbours than the shared-memory lists
    hold), 400 hyperedges through hub 2 alone (light pairs: stars), a few
    of 65-100 members whose members past position 63 are shared with small
    hyperedges, size-1 and size-2 hyperedges on the hubs, and random ones."""
    rows = [[0, 1, 10 + int(x)] for x in rng.choice(3000, size=300, replace=False)]
    rows += [[2] + sorted(rng.choice(np.arange(4000, 9000), size=int(rng.integers(1, 5)), replace=False).tolist())
             for _ in range(400)]
    rows += [[2], [2], [0], [2, 5], [2, 6], [0, 1]]
    for k in (65, 80, 100):
        big = sorted(rng.choice(np.arange(9000, 9400), size=k, replace=False).tolist())
        rows.append(big)
        for p in (0, 30, 63, 64, k - 1):
            rows.append([big[p], 9500 + int(rng.integers(0, 50))])
        rows.append([big[70 % k], big[3], 2])
    rows += [sorted(rng.choice(9600, size=int(rng.integers(2, 7)), replace=False).tolist()) for _ in range(800)]
    return rows


@pytest.mark.parametrize("seed", range(3))
def test_grouped_walk_equals_plain_walk_and_oracle(ctx, seed):
    """The static count with the shared-member groups counted in bulk (the
    default) and with every oriented entry visited give the oracle's counts,
    on a graph made to reach every branch of the grouped walk and on
    config-2-law graphs, under the default and all-block schedules."""
    from ipdps26_b200 import engine, gen

    rng = np.random.default_rng(900 + seed)
    cases = [(*csr(_heavy_rich_rows(rng)), 9700)]
    h = gen.static(gen.config2(seed=40 + seed, n_nodes=4000, n_edges=8000, q=40.0))
    cases.append((h.offsets, h.members, h.n_nodes))
    for off, mem, n_nodes in cases:
        want = oracle.static30(off, mem, n_nodes)
        with engine.Graph(ctx, off, mem, n_nodes) as g:
            for sched in ((128, 2048), (0, 0)):
                g.set_schedule(*sched)
                for on in (True, False):
                    g.set_static_groups(on)
                    assert g.count_static30().tolist() == want.tolist(), (sched, on)


def test_oriented_rows_longer_than_the_table(ctx):
    """A centre with more than 4,096 neighbours ranked above it is counted
    without its shared-memory table (a filter in that memory, then a search of
    its H2H row): hyperedge 0 = {0..9} and 4,200 hyperedges {z, i mod 10,
    1000 + i} of equal degree above it. Checked against the touched-triple
    count of every hyperedge (other kernels, a count of the same triples)."""
    from ipdps26_b200 import engine

    z = 999
    rows = [list(range(10))] + [sorted({z, i % 10, 1000 + i}) for i in range(4200)]
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, 1000 + 4200) as g:
        g.set_schedule(128, 2048)
        full = g.count_static30()
        every = g.count_touching30(np.arange(len(rows), dtype=np.uint32))
        assert full.tolist() == every.tolist()
        assert int(full.sum()) > 0
