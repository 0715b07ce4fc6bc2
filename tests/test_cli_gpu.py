"""The command-line driver on the GPU: its printed counts equal the oracle's
for generated, MoCHy-format and THyMe-format inputs."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "ipdps26_b200" / "hmotif"


def _run(*args):
    r = subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _bins(out, title):
    m = re.search(re.escape(title) + r" \(30 bins\): ([-\d ]+)", out)
    assert m, out
    return [int(x) for x in m.group(1).split()]


def _motifs(out, n):
    got = dict((int(a), int(b)) for a, b in re.findall(r"^motif (\d+): (\d+)$", out, flags=re.M))
    return [got[i] for i in range(1, n + 1)]


def test_generate_mode_matches_oracle(tmp_path):
    from ipdps26_b200 import formats
    from oracle import oracle

    out = _run("300", "6", "1", "120", "4096", "-totalChanges", "40", "--seed=7", f"--input-dir={tmp_path}",
               "--save-generated=g.txt")
    h = formats.read(tmp_path / "g.txt", "escher")
    assert h.n_edges == 300
    before = _bins(out, "Motif counts")
    assert before == oracle.static30(h.offsets, h.members, 120).tolist()
    delta = _bins(out, "Motif delta counts")
    after = _bins(out, "Motif counts after the batch")
    assert [a - b for a, b in zip(after, before)] == delta
    assert "deletes: 20, inserts: 20" in out


def test_mochy_input_matches_oracle(tmp_path):
    from ipdps26_b200 import formats, gen
    from oracle import oracle

    h = gen.static(gen.params(11, 400, 800, 2, 12, 2.5, 1.2, 0.0))
    formats.write(h, tmp_path / "m.txt", "mochy")
    out = _run("4096", "--input=m.txt", f"--input-dir={tmp_path}", "--input-format=mochy", "--mochy", "--no-update")
    n_nodes = int(h.members.max()) + 1
    c30 = oracle.static30(h.offsets, h.members, n_nodes)
    assert _bins(out, "Motif counts") == c30.tolist()
    assert _motifs(out, 26) == oracle.to26(c30).tolist()


def test_thyme_input_temporal_matches_oracle(tmp_path):
    from ipdps26_b200 import formats, gen
    from oracle import oracle

    h = gen.temporal(gen.params(4, 300, 1500, 2, 8, 2.5, 1.2, 0.0, dedupe=False), burst_rate=1e-3,
                     events_per_burst=20, gap_mean=5.0, span=200_000)
    formats.write(h, tmp_path / "t.txt", "thyme")
    out = _run("4096", "--input=t.txt", f"--input-dir={tmp_path}", "--input-format=thyme", "--temporal-delta=5000")
    want = oracle.temporal96(h.offsets, h.members, h.timestamps, 5000)
    assert _motifs(out, 96) == want.tolist()


def _csr(rows):
    off = np.zeros(len(rows) + 1, np.uint64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return off, np.array([v for r in rows for v in r], np.uint32)


def _delta(new, old):
    return (np.asarray(new).astype(np.int64) - np.asarray(old).astype(np.int64)).tolist()


def test_temporal_synthetic_window_with_deltas(tmp_path):
    """--temporal --temporal-synthetic --temporal-deltas: the reference's fixed
    window, its newer window with the deltas file applied to the newest
    layer, against the oracle's strictly increasing count."""
    from oracle import oracle

    d = tmp_path / "updates_synth.txt"
    d.write_text("A 2 1 4\nR 3 1\n")
    out = _run("8", "5", "1", "100", "4096", "--seed=3", f"--input-dir={tmp_path}", "--temporal",
               "--temporal-synthetic", f"--temporal-deltas={d}")
    L = [[0, 1], [1, 2], [0, 2]]
    newest = [[0, 1], [0, 1, 2, 3], [1, 2]]  # {1,2},{2,3}+{1,4},{1,2,3}-{1}, vertex v as node v - 1
    old = oracle.strictinc30([_csr(L)] * 3)
    new = oracle.strictinc30([_csr(L), _csr(L), _csr(newest)])
    assert _bins(out, "Temporal strict-inc counts") == old.tolist()
    assert _bins(out, "Temporal strict-inc delta") == _delta(new, old)
    assert any(_delta(new, old))


def test_temporal_window_after_the_batch(tmp_path):
    """--temporal on a generated graph: all layers hold the graph, then the
    newest layer holds it after a deletion-only batch (deleted rows empty)."""
    from ipdps26_b200 import formats
    from oracle import oracle

    out = _run("60", "6", "1", "40", "4096", "--seed=5", f"--input-dir={tmp_path}", "--save-generated=g.txt",
               "-totalChanges", "10", "-insertionPercentage", "0", "-deletionPercentage", "100", "--temporal")
    assert "deletes: 10, inserts: 0" in out
    h = formats.read(tmp_path / "g.txt", "escher")
    rows = [list(h.edge(i)) for i in range(h.n_edges)]
    upd = [r if i < h.n_edges - 10 else [] for i, r in enumerate(rows)]
    old = oracle.strictinc30([_csr(rows)] * 3)
    new = oracle.strictinc30([_csr(rows), _csr(rows), _csr(upd)])
    assert _bins(out, "Temporal strict-inc counts") == old.tolist()
    assert _bins(out, "Temporal strict-inc delta") == _delta(new, old)
    assert old.sum() > 0
