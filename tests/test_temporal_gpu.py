"""Temporal 96-motif counts on the GPU against THyMe's own outputs (golden
fixtures) and the CPU oracle."""
import numpy as np
import pytest

from oracle import oracle, refdata
from tests.helpers import csr, digest, load_golden, random_graph, temporal_case

pytestmark = pytest.mark.gpu


def test_temporal_on_thyme_email_enron(ctx):
    """THyMe's dataset through the GPU at delta = 86,400,000: the total (127,357
    in all three of THyMe's shipped exact results) and the per-static-class
    sums, which do not depend on tie-breaking; and, with ties ordered by input
    position on both sides, every one of the 96 counts equals the oracle."""
    from ipdps26_b200 import engine

    rec = load_golden("temporal")["email-Enron"]
    p = refdata.path("email-Enron")
    if p is None:
        pytest.skip("reference dataset not present (oracle/build_ref.sh copies it)")
    assert refdata.sha256(p) == rec["file_sha256"]
    off, mem, times, n_nodes = refdata.read_thyme(p)
    with engine.Graph(ctx, off, mem, n_nodes, times) as g:
        got = g.count_temporal(rec["delta"])
    assert int(got.sum()) == rec["total"]
    assert refdata.per_static(got) == rec["per_static"]
    assert got.tolist() == oracle.temporal96(off, mem, times, rec["delta"]).tolist()


@pytest.mark.parametrize("name", sorted(k for k, v in load_golden("temporal").items() if "params" in v))
def test_temporal_matches_thyme_golden(ctx, name):
    from ipdps26_b200 import engine

    rec = load_golden("temporal")[name]
    h = temporal_case(rec["params"])
    assert digest(h) == rec["sha256"]
    with engine.Graph.from_hypergraph(ctx, h) as g:
        for d, want in rec["counts96"].items():
            assert g.count_temporal(int(d)).tolist() == want, d


@pytest.mark.parametrize("seed", range(6))
def test_temporal_matches_oracle_random(ctx, seed):
    from ipdps26_b200 import engine

    rng = np.random.default_rng(50 + seed)
    n_nodes = int(rng.integers(6, 30))
    off, mem = random_graph(rng, int(rng.integers(5, 120)), n_nodes, int(rng.integers(2, 6)), p_repeat=0.2)
    rows = [mem[off[i]:off[i + 1]].tolist() for i in range(len(off) - 1)]
    for i in range(0, len(rows), 4):  # repeated node-sets
        rows[i] = rows[max(0, i - 2)]
    off, mem = csr(rows)
    times = np.cumsum(rng.integers(1, 30, size=len(rows))).astype(np.int64)
    perm = rng.permutation(len(rows))  # input order differs from time order
    rows = [rows[i] for i in perm]
    times = times[perm]
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, n_nodes, times) as g:
        for delta in (0, 20, 100, 10_000):
            want = oracle.temporal96(off, mem, times, delta)
            assert g.count_temporal(delta).tolist() == want.tolist(), delta


def test_temporal_graph_is_not_static(ctx):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HmError

    off, mem = csr([[0, 1], [1, 2]])
    with engine.Graph(ctx, off, mem, 3, np.array([1, 2], np.int64)) as g:
        with pytest.raises(HmError) as e:
            g.count_static30()
        assert e.value.status == -7
        with pytest.raises(HmError):
            g.apply_batch([0])
        with pytest.raises(HmError) as e:
            g.count_temporal(-1)
        assert e.value.status == -1


def test_temporal_c4_laws(ctx):
    from ipdps26_b200 import engine, gen

    h = gen.temporal(gen.config4(seed=8, n_nodes=1500, n_edges=3000), span=600_000)
    with engine.Graph.from_hypergraph(ctx, h) as g:
        for delta in (1000, 10_000):
            want = oracle.temporal96(h.offsets, h.members, h.timestamps, delta)
            assert g.count_temporal(delta).tolist() == want.tolist(), delta


@pytest.mark.parametrize("seed", range(8))
def test_temporal_with_equal_times_matches_oracle(ctx, seed):
    """Inputs where many events share a timestamp, and node-sets repeat: the
    GPU and the oracle follow one tie rule (events in input order; a tie
    between two occurrences counts as c before b, b the node-set met first
    in the input), so all 96 counts agree."""
    from ipdps26_b200 import engine

    rng = np.random.default_rng(700 + seed)
    for _ in range(25):
        n_nodes = int(rng.integers(3, 10))
        off, mem = random_graph(rng, int(rng.integers(3, 30)), n_nodes, 4)
        rows = [mem[off[i]:off[i + 1]].tolist() for i in range(len(off) - 1)]
        for i in range(0, len(rows), 3):
            rows[i] = rows[max(0, i - 1)]
        off, mem = csr(rows)
        times = rng.integers(0, 5, size=len(rows)).astype(np.int64)
        with engine.Graph(ctx, off, mem, n_nodes, times) as g:
            for delta in (0, 1, 3, 10):
                want = oracle.temporal96(off, mem, times, delta)
                assert g.count_temporal(delta).tolist() == want.tolist(), (rows, times.tolist(), delta)


def spokes_and_centres(rng, nodes_per_centre, spokes_per_node, centres):
    """Small "spoke" events {v, unique node} and, after them, large "centre"
    events over the spokes' shared nodes: a centre's window holds about
    nodes_per_centre * spokes_per_node neighbours while the spokes' own
    windows stay small."""
    n_shared = nodes_per_centre + 20 * (centres - 1)
    spokes = [[v, 100_000 + j] for j, v in enumerate(rng.permutation(np.repeat(np.arange(1, n_shared + 1),
                                                                                   spokes_per_node)))]
    cents = [list(range(1 + 20 * c, 1 + 20 * c + nodes_per_centre)) for c in range(centres)]
    rows = spokes + cents
    off, mem = csr(rows)
    times = np.arange(len(rows), dtype=np.int64)
    return off, mem, times, 100_000 + len(spokes)


def test_temporal_wide_windows_take_the_deferred_launch(ctx):
    """Events with more than 1,024 window neighbours are set aside by the first
    launch and counted by the second (8,192-slot table): centres with about
    1,200 neighbours, against the oracle."""
    from ipdps26_b200 import engine

    rng = np.random.default_rng(77)
    off, mem, times, n_nodes = spokes_and_centres(rng, 100, 12, 3)
    with engine.Graph(ctx, off, mem, n_nodes, times) as g:
        got = g.count_temporal(1_000_000)
    assert got.tolist() == oracle.temporal96(off, mem, times, 1_000_000).tolist()


def test_temporal_window_limit_is_an_error(ctx):
    """More than 4,096 neighbours of one event inside its window is reported
    (HM_ERR_LIMIT), not counted wrong, and the graph stays usable."""
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_LIMIT, HmError

    rng = np.random.default_rng(78)
    off, mem, times, n_nodes = spokes_and_centres(rng, 250, 17, 1)
    with engine.Graph(ctx, off, mem, n_nodes, times) as g:
        with pytest.raises(HmError) as e:
            g.count_temporal(1_000_000)
        assert e.value.status == HM_ERR_LIMIT
        assert g.count_temporal(10).tolist() == oracle.temporal96(off, mem, times, 10).tolist()
