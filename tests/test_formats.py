"""Reference file formats (hm_hostgraph_read / hm_hostgraph_write) and the
command-line driver's argument handling, on the CPU."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.helpers import random_graph

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "ipdps26_b200" / "hmotif"


def _graph(seed=0, n=40, nodes=30, kmax=6, times=False):
    from ipdps26_b200.gen import Hypergraph

    rng = np.random.default_rng(seed)
    off, mem = random_graph(rng, n, nodes, kmax)
    ts = np.cumsum(rng.integers(1, 50, size=n)).astype(np.int64) if times else None
    return Hypergraph(off, mem, nodes, ts)


def _rows(h):
    return [h.members[h.offsets[e]:h.offsets[e + 1]].tolist() for e in range(h.n_edges)]


def _dedup(r):
    out = []
    for v in r:
        if v not in out:
            out.append(v)
    return out


@pytest.mark.parametrize("fmt", ["escher", "mochy", "thyme"])
def test_round_trip(tmp_path, fmt):
    from ipdps26_b200 import formats

    h = _graph(1, times=(fmt == "thyme"))
    p = tmp_path / "g.txt"
    formats.write(h, p, fmt)
    g = formats.read(p, fmt)
    assert _rows(g) == [_dedup(r) for r in _rows(h)]
    assert g.n_nodes == int(h.members.max()) + 1
    if fmt == "thyme":
        assert g.timestamps.tolist() == h.timestamps.tolist()


def test_written_text_matches_reference_writers(tmp_path):
    """MoCHy and THyMe files as the reference programs read them (the same
    text the runner of the reference counters writes), ESCHER 1-based."""
    from ipdps26_b200 import formats
    from oracle import ref_runner as rr

    h = _graph(2, times=True)
    formats.write(h, tmp_path / "m.txt", "mochy")
    rr.write_mochy(tmp_path / "m_ref.txt", h.offsets, h.members)
    assert (tmp_path / "m.txt").read_text() == (tmp_path / "m_ref.txt").read_text()
    formats.write(h, tmp_path / "t.txt", "thyme")
    rr.write_thyme(tmp_path / "t_ref.txt", h.offsets, h.members, h.timestamps)
    assert (tmp_path / "t.txt").read_text() == (tmp_path / "t_ref.txt").read_text()
    formats.write(h, tmp_path / "e.txt", "escher")
    lines = (tmp_path / "e.txt").read_text().splitlines()
    assert lines == [" ".join(str(v + 1) for v in r) for r in _rows(h)]


def test_escher_reader_rules(tmp_path):
    from ipdps26_b200 import formats
    from ipdps26_b200._lib import HM_ERR_INVALID, HmError

    p = tmp_path / "e.txt"
    p.write_text("# a comment\n3 1 2\n\n5  4\n# another\n7\n")
    g = formats.read(p, "escher")
    assert _rows(g) == [[2, 0, 1], [4, 3], [6]]
    assert g.n_nodes == 7
    for bad in ("1 0 2\n", "1 -3\n", "1 x\n"):
        p.write_text(bad)
        with pytest.raises(HmError) as e:
            formats.read(p, "escher")
        assert e.value.status == HM_ERR_INVALID


def test_mochy_and_thyme_reader_rules(tmp_path):
    from ipdps26_b200 import formats
    from ipdps26_b200._lib import HmError

    p = tmp_path / "m.txt"
    p.write_text("0,4,4,2\n3\n1,0\n")
    assert _rows(formats.read(p, "mochy")) == [[0, 4, 2], [3], [1, 0]]
    p.write_text("0,,1\n")
    with pytest.raises(HmError):
        formats.read(p, "mochy")
    t = tmp_path / "t.txt"
    t.write_text("0,1\t10\n2,1\t11.0\n")
    g = formats.read(t, "thyme")
    assert g.timestamps.tolist() == [10, 11]
    t.write_text("0,1\t10.5\n")
    with pytest.raises(HmError):
        formats.read(t, "thyme")
    t.write_text("0,1 10\n")
    with pytest.raises(HmError):
        formats.read(t, "thyme")
    with pytest.raises(HmError):
        formats.read(tmp_path / "missing.txt", "mochy")


def _cli(*args):
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=60)


@pytest.mark.skipif(not CLI.exists(), reason="command-line driver not built")
@pytest.mark.parametrize("args, msg", [
    ((), "Usage"),
    (("5", "3", "1", "10"), "generate mode expects"),
    (("5", "3", "10", "1", "4096"), "min_vertex_id must be less"),
    (("5", "0", "1", "10", "4096"), "positive integers"),
    (("4096", "--input=x.txt", "--input-format=csv"), "unknown input format"),
    (("4096", "--input=x.txt", "--temporal-delta=10"), "needs --input-format=thyme"),
    (("5", "3", "1", "10", "4096", "-totalChanges", "0"), "totalChanges must be a positive integer"),
    (("5", "3", "1", "10", "4096", "-insertionPercentage", "0", "-deletionPercentage", "0"), "sum must be > 0"),
    (("1", "2", "3", "--input=f.txt"), "input mode expects"),
])
def test_cli_rejects_bad_arguments(args, msg):
    r = _cli(*args)
    assert r.returncode == 1
    assert msg in r.stderr
