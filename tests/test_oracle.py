"""The CPU oracle (C restatement of MoCHy / THyMe exact) against the
reference programs' own outputs (golden fixtures) and against brute force."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle, refdata
from tests.helpers import csr, digest, load_golden, random_graph, static_case, temporal_case

ROOT = Path(__file__).resolve().parents[1]
SYNTHETIC_TEMPORAL = sorted(k for k, v in load_golden("temporal").items() if "params" in v)


@pytest.mark.parametrize("name", sorted(load_golden("static")))
def test_static_oracle_matches_mochy(name):
    rec = load_golden("static")[name]
    if name == "dblp":
        p = refdata.path("dblp")
        if p is None:
            pytest.skip("reference dataset not present (oracle/build_ref.sh copies it)")
        assert hashlib.sha256(p.read_bytes()).hexdigest() == rec["file_sha256"]
        off, mem, n_nodes = refdata.read_mochy(p)
    else:
        if rec["n_edges"] > 3000:
            pytest.skip("large case: covered by the GPU parity test")
        h = static_case(rec["params"])
        assert digest(h) == rec["sha256"], "generator output changed"
        off, mem, n_nodes = h.offsets, h.members, h.n_nodes
    got = oracle.to26(oracle.static30(off, mem, n_nodes))
    assert got.tolist() == rec["counts26"]


@pytest.mark.parametrize("name", SYNTHETIC_TEMPORAL)
def test_temporal_oracle_matches_thyme(name):
    rec = load_golden("temporal")[name]
    if rec["n_events"] > 2000:
        pytest.skip("large case: covered by the GPU parity test")
    h = temporal_case(rec["params"])
    assert digest(h) == rec["sha256"], "generator output changed"
    for d, want in rec["counts96"].items():
        got = oracle.temporal96(h.offsets, h.members, h.timestamps, int(d))
        assert got.tolist() == want, d


def test_temporal_oracle_on_thyme_email_enron():
    """THyMe's own dataset and shipped results (delta = 86,400,000): the
    dataset has ties in time, which THyMe breaks at random, so the check is
    on what ties cannot change: the total and the sum per static class, which
    all three of THyMe's exact programs agree on."""
    rec = load_golden("temporal")["email-Enron"]
    p = refdata.path("email-Enron")
    if p is None:
        pytest.skip("reference dataset not present (oracle/build_ref.sh copies it)")
    assert refdata.sha256(p) == rec["file_sha256"]
    off, mem, times, _ = refdata.read_thyme(p)
    got = oracle.temporal96(off, mem, times, rec["delta"])
    assert int(got.sum()) == rec["total"] == 127357
    assert refdata.per_static(got) == rec["per_static"]
    for k in ("thyme", "thymeP", "dp"):  # the fixture agrees with every shipped result file
        rp = refdata.path(f"email-Enron-{k}")
        if rp is not None:
            assert refdata.per_static(refdata.read_thyme_result(rp)[1]) == rec["per_static"]


@pytest.mark.parametrize("seed", range(6))
def test_static_oracle_matches_brute_force(seed):
    rng = np.random.default_rng(seed)
    off, mem = random_graph(rng, 45, 30, 7, p_repeat=0.3)
    n_nodes = 30
    a = oracle.static30(off, mem, n_nodes)
    b = oracle.static30_brute(off, mem)
    assert a.tolist() == b.tolist()


@pytest.mark.parametrize("seed", range(4))
def test_temporal_oracle_matches_brute_force(seed):
    rng = np.random.default_rng(100 + seed)
    off, mem = random_graph(rng, 40, 12, 4)
    # repeat some node-sets (THyMe's motifs 87-96)
    rows = [mem[off[i]:off[i + 1]].tolist() for i in range(len(off) - 1)]
    for i in range(0, len(rows), 5):
        rows[i] = rows[max(0, i - 3)]
    off, mem = csr(rows)
    times = np.cumsum(rng.integers(1, 20, size=len(rows))).astype(np.int64)
    for delta in (15, 60, 400):
        a = oracle.temporal96(off, mem, times, delta)
        b = oracle.temporal96_brute(off, mem, times, delta)
        assert a.tolist() == b.tolist()
        assert a[86:].sum() > 0 or delta == 15


def test_class_rules_agree_with_oracle():
    from ipdps26_b200 import engine

    L = oracle.lib()
    for p in range(128):
        assert engine.classify_static(p) == L.hmo_static_class_bits(p)
        assert engine.classify_temporal(p) == L.hmo_temporal_class_bits(p)
    # 30 static classes and 96 temporal motifs are each hit by some pattern
    assert {engine.classify_static(p) for p in range(128)} - {-1} == set(range(30))
    assert {engine.classify_temporal(p) for p in range(128)} - {-1} == set(range(96))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_vertex_triads_match_reference_programs(seed, tmp_path):
    """The restated type1/2/3 counts equal the reference's own counters
    (temporalDynamicHMotif/src/type{1,2,3}.cpp, built by build_ref.sh)."""
    import subprocess

    from oracle import oracle, ref_runner as rr

    exe = [ROOT / "oracle" / "_ref" / f"type{t}" for t in (1, 2, 3)]
    if not all(e.exists() for e in exe):
        pytest.skip("reference type counters not built (reference tree absent)")
    rng = np.random.default_rng(seed)
    off, mem = random_graph(rng, 150, 50, 10)
    g = tmp_path / "g.txt"
    rr.write_mochy(g, off, mem)
    ref = [int(subprocess.run([str(e), str(g)], capture_output=True, text=True, check=True).stdout.split()[-1])
           for e in exe]
    assert oracle.vertex_triads(off, mem).tolist() == ref


def test_strictinc_hand_case():
    """One closed triple across the layers (older {0,1}, middle {1,2},
    newest {0,2}): pairwise overlaps 1, no shared node; ids in order."""
    from oracle import oracle

    L0 = (np.array([0, 2], np.uint64), np.array([0, 1], np.uint32))
    L1 = (np.array([0, 1, 3], np.uint64), np.array([9, 1, 2], np.uint32))
    L2 = (np.array([0, 1, 2, 4], np.uint64), np.array([8, 7, 0, 2], np.uint32))
    c = oracle.strictinc30([L0, L1, L2])
    assert c.sum() == 1
    assert c[oracle.lib().hmo_static_class(2, 2, 2, 1, 1, 1, 0)] == 1
    # the same triple with the newest one earlier than the middle one: none
    L2b = (np.array([0, 2, 3, 4], np.uint64), np.array([0, 2, 8, 7], np.uint32))
    assert oracle.strictinc30([L0, L1, L2b]).sum() == 0
