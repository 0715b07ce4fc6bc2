"""Seeded generators: deterministic, sorted unique members, laws respected."""
import numpy as np

from ipdps26_b200 import gen


def test_static_deterministic_sorted_unique():
    p = gen.config1(seed=7, n_nodes=500, n_edges=800)
    a, b = gen.static(p), gen.static(p)
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.members, b.members)
    assert a.n_edges == 800
    seen = set()
    for e in range(a.n_edges):
        r = a.edge(e)
        assert 2 <= len(r) <= 25
        assert np.all(np.diff(r.astype(np.int64)) > 0)
        assert r.max() < 500
        seen.add(tuple(r.tolist()))
    assert len(seen) == 800  # duplicates were redrawn


def test_popularity_offset_flattens_hubs():
    a = gen.static(gen.config2(seed=1, n_nodes=20000, n_edges=20000, q=0.0))
    b = gen.static(gen.config2(seed=1, n_nodes=20000, n_edges=20000, q=1000.0))
    assert np.bincount(a.members).max() > 3 * np.bincount(b.members).max()


def test_temporal_strictly_increasing():
    h = gen.temporal(gen.config4(seed=3, n_nodes=2000, n_edges=5000), span=1_000_000)
    assert h.timestamps is not None and len(h.timestamps) == 5000
    assert np.all(np.diff(h.timestamps) > 0)
    assert h.timestamps[-1] <= 1_000_000 + 5000


def test_batch_generator():
    p = gen.config1(seed=0, n_nodes=500, n_edges=800)
    live = np.arange(800, dtype=np.uint32)
    d, ins = gen.batch(p, 99, live, 100, 0.8)
    assert len(d) == 20 and np.all(np.diff(d.astype(np.int64)) > 0) and d.max() < 800
    assert ins.n_edges == 80
    d2, ins2 = gen.batch(p, 99, live, 100, 0.8)
    assert np.array_equal(d, d2) and np.array_equal(ins.members, ins2.members)
