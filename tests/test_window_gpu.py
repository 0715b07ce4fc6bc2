"""Three-layer temporal window and its strictly increasing count against the
oracle's restatement (brute force over all i < j < k)."""
import numpy as np
import pytest

from tests.helpers import random_graph

pytestmark = pytest.mark.gpu


def _layers(seed, n=(60, 70, 80), nodes=40, kmax=7):
    rng = np.random.default_rng(seed)
    return [random_graph(rng, m, nodes, kmax) for m in n]


def _rows(off, mem):
    return [list(mem[off[e]:off[e + 1]]) for e in range(len(off) - 1)]


def _csr(rows):
    off = np.zeros(len(rows) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    mem = np.array([v for r in rows for v in r], np.uint32)
    return off, mem


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_count_matches_oracle(ctx, seed):
    from ipdps26_b200 import engine
    from oracle import oracle

    layers = _layers(seed)
    with engine.Window(ctx, 40) as w:
        for l, (off, mem) in enumerate(layers):
            w.set_layer(l, off, mem)
        got = w.count30()
    want = oracle.strictinc30(layers)
    assert got.tolist() == want.tolist()
    assert want.sum() > 0


def test_rotation_fill_unfill_and_deltas(ctx, tmp_path):
    from ipdps26_b200 import engine
    from oracle import oracle

    a, b, c, d = _layers(9, n=(50, 50, 50, 50))
    with engine.Window(ctx, 40) as w:
        w.set_layer(engine.OLDER, *a)
        w.set_layer(engine.MIDDLE, *b)
        w.set_layer(engine.NEWEST, *c)
        assert w.count30().tolist() == oracle.strictinc30([a, b, c]).tolist()
        # ring: Older <- Middle <- Newest; the old Older becomes Newest, then is replaced
        w.rotate()
        w.reset_layer(engine.NEWEST)
        assert w.layer_size(engine.NEWEST) == 0
        assert w.count30().sum() == 0
        w.set_layer(engine.NEWEST, *d)
        assert w.count30().tolist() == oracle.strictinc30([b, c, d]).tolist()
        # fill / unfill on the newest layer
        rows = _rows(*d)
        w.fill(engine.NEWEST, [3, 7], [[1, 2, 39], [0]])
        w.unfill(engine.NEWEST, [5], [rows[5][:1]])
        rows[3] = sorted(set(rows[3]) | {1, 2, 39})
        rows[7] = sorted(set(rows[7]) | {0})
        rows[5] = sorted(set(rows[5]) - set(rows[5][:1]))
        assert w.count30().tolist() == oracle.strictinc30([b, c, _csr(rows)]).tolist()
        # the reference's delta file: 1-based hyperedges and vertices
        p = tmp_path / "deltas.txt"
        p.write_text("A 1 5 6\nR 2 %d\n\nA 10 40\n" % (rows[1][0] + 1))
        w.apply_deltas_file(p)
        rows[0] = sorted(set(rows[0]) | {4, 5})
        rows[1] = sorted(set(rows[1]) - {rows[1][0]})
        rows[9] = sorted(set(rows[9]) | {39})
        assert w.count30().tolist() == oracle.strictinc30([b, c, _csr(rows)]).tolist()


def test_bad_inputs_change_nothing(ctx, tmp_path):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_INVALID, HM_ERR_NOT_LIVE, HmError

    a, b, c = _layers(4, n=(20, 20, 20))
    with engine.Window(ctx, 40) as w:
        for l, layer in enumerate((a, b, c)):
            w.set_layer(l, *layer)
        before = w.count30().tolist()
        with pytest.raises(HmError) as e:
            w.fill(engine.NEWEST, [25], [[1]])
        assert e.value.status == HM_ERR_NOT_LIVE
        with pytest.raises(HmError) as e:
            w.fill(engine.NEWEST, [2], [[40]])
        assert e.value.status == HM_ERR_INVALID
        with pytest.raises(HmError):
            w.set_layer(3, *a)
        p = tmp_path / "bad.txt"
        p.write_text("X 1 2\n")
        with pytest.raises(HmError):
            w.apply_deltas_file(p)
        assert w.count30().tolist() == before


REF_STRICTINC = __import__("pathlib").Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "strictinc"


def _reference_layers(seed, sizes=(1, 2, 3, 5, 6, 7)):
    """Three random layers inside the reference counter's own limits: no
    hyperedge size a multiple of 4 (its payload then lacks an end marker)
    and few enough hyperedges that no middle one has 1024 candidates."""
    rng = np.random.default_rng(seed)
    n_nodes = int(rng.integers(12, 45))
    layers = []
    for _ in range(3):
        m = int(rng.integers(20, 120))
        rows = [sorted(rng.choice(n_nodes, size=min(int(rng.choice(sizes)), n_nodes), replace=False).tolist())
                for _ in range(m)]
        layers.append(rows)
    return n_nodes, layers


@pytest.mark.parametrize("seed", range(6))
def test_strictinc_matches_the_reference_counter(ctx, seed, tmp_path):
    """The reference's own temporalStrictIncAdjKernel (built from its sources
    into oracle/_ref/strictinc by build_ref.sh, run on this GPU) against
    hm_window_count30 and the oracle, bin for bin."""
    import subprocess

    from ipdps26_b200 import engine
    from oracle import oracle

    if not REF_STRICTINC.exists():
        pytest.skip("reference counter not built (oracle/build_ref.sh needs the reference tree and nvcc)")
    n_nodes, layers = _reference_layers(seed)
    f = tmp_path / "layers.txt"
    with open(f, "w") as fh:  # vertices are 1-based in the reference's stores
        fh.write(f"{n_nodes}\n")
        for rows in layers:
            fh.write(f"{len(rows)}\n")
            for r in rows:
                fh.write(f"{len(r)} {' '.join(str(v + 1) for v in r)}\n")
    r = subprocess.run([str(REF_STRICTINC), str(f)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("strictinc30:")]
    assert line, r.stdout[-2000:]
    ref = [int(x) for x in line[-1].split()[1:]]
    assert len(ref) == 30
    csrs = [_csr(rows) for rows in layers]
    with engine.Window(ctx, n_nodes) as w:
        for l, (off, mem) in enumerate(csrs):
            w.set_layer(l, off, mem)
        got = w.count30()
    assert sum(ref) > 0
    assert got.tolist() == ref
    assert oracle.strictinc30(csrs).tolist() == ref
