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
