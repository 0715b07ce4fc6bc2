"""Generates the golden fixtures: outputs of the reference's OWN counters.

Each case is a seeded synthetic input (regenerated by the tests from the
recorded parameters; its SHA-256 is recorded too) run through the reference
programs compiled from the reference sources by oracle/build_ref.sh:
  static   -> MoCHy main_exact and main_exact_par (26 counts)
  temporal -> THyMe main_thyme and main_thymeP (96 counts)
The MoCHy sample dataset shipped with the reference (dblp_graph.txt) is
recorded by its hash and counts only; its test runs where the reference tree
is present.

    python tests/golden/make_golden.py [--only NAME ...]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ipdps26_b200 import gen  # noqa: E402
from oracle import ref_runner as rr  # noqa: E402
from oracle import refdata  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest(h) -> str:
    m = hashlib.sha256()
    m.update(np.ascontiguousarray(h.offsets, np.uint64).tobytes())
    m.update(np.ascontiguousarray(h.members, np.uint32).tobytes())
    if h.timestamps is not None:
        m.update(np.ascontiguousarray(h.timestamps, np.int64).tobytes())
    return m.hexdigest()


# name -> (generator params kwargs of gen.params)
STATIC_CASES = {}
for s in range(5):
    STATIC_CASES[f"tiny-c1-{s}"] = dict(seed=s, n_nodes=60, n_edges=80, k_min=2, k_max=25, size_exp=2.5, pop_exp=1.2,
                                        pop_offset=0.0)
for s in range(2):
    STATIC_CASES[f"c1law-2k-{s}"] = dict(seed=10 + s, n_nodes=1000, n_edges=2000, k_min=2, k_max=25, size_exp=2.5,
                                         pop_exp=1.2, pop_offset=0.0)
STATIC_CASES["c2law-3k"] = dict(seed=21, n_nodes=3000, n_edges=3000, k_min=2, k_max=100, size_exp=2.2, pop_exp=1.1,
                                pop_offset=3.0)
STATIC_CASES["c2law-10k-flat"] = dict(seed=22, n_nodes=20000, n_edges=10000, k_min=2, k_max=100, size_exp=2.2,
                                      pop_exp=1.1, pop_offset=1000.0)
STATIC_CASES["wide-overlaps"] = dict(seed=23, n_nodes=120, n_edges=400, k_min=2, k_max=40, size_exp=1.5, pop_exp=0.8,
                                     pop_offset=0.0)
STATIC_CASES["size1-and-dups"] = dict(seed=24, n_nodes=50, n_edges=300, k_min=1, k_max=6, size_exp=1.5, pop_exp=1.0,
                                      pop_offset=0.0, dedupe=False)

TEMPORAL_CASES = {}
for s in range(4):
    TEMPORAL_CASES[f"tiny-c4-{s}"] = dict(
        gen=dict(seed=s, n_nodes=40, n_edges=60, k_min=2, k_max=20, size_exp=2.5, pop_exp=1.2, pop_offset=0.0,
                 dedupe=False),
        burst=dict(burst_rate=1e-2, events_per_burst=10, gap_mean=5.0, span=2000), deltas=[50, 300, 5000])
TEMPORAL_CASES["c4law-20k"] = dict(
    gen=dict(seed=31, n_nodes=8000, n_edges=20000, k_min=2, k_max=20, size_exp=2.5, pop_exp=1.2, pop_offset=0.0,
             dedupe=False),
    burst=dict(burst_rate=1e-4, events_per_burst=50, gap_mean=20.0, span=4_000_000), deltas=[1000, 10000, 100000])


def static_graph(p):
    kw = dict(p)
    dedupe = kw.pop("dedupe", True)
    return gen.static(gen.params(dedupe=dedupe, **kw))


def temporal_graph(c):
    kw = dict(c["gen"])
    dedupe = kw.pop("dedupe", False)
    return gen.temporal(gen.params(dedupe=dedupe, **kw), **c["burst"])


FULL_CASES = {
    # config 1 exactly as specified (MoCHy main_exact_par on all host cores)
    "config1-full": dict(kind="static", params=dict(seed=0, n_nodes=10000, n_edges=20000, k_min=2, k_max=25,
                                                    size_exp=2.5, pop_exp=1.2, pop_offset=0.0)),
    # config 4 as specified (THyMe+ main_thymeP on all host cores), smallest window
    "config4-full-d1000": dict(kind="temporal", params=dict(
        gen=dict(seed=3, n_nodes=200000, n_edges=500000, k_min=2, k_max=20, size_exp=2.5, pop_exp=1.2,
                 pop_offset=0.0, dedupe=False),
        burst=dict(burst_rate=1e-4, events_per_burst=50, gap_mean=20.0, span=100_000_000), deltas=[1000])),
    # the same stream at the two wider windows of config 4
    "config4-full-d10000": dict(kind="temporal", params=dict(
        gen=dict(seed=3, n_nodes=200000, n_edges=500000, k_min=2, k_max=20, size_exp=2.5, pop_exp=1.2,
                 pop_offset=0.0, dedupe=False),
        burst=dict(burst_rate=1e-4, events_per_burst=50, gap_mean=20.0, span=100_000_000), deltas=[10000])),
    "config4-full-d100000": dict(kind="temporal", params=dict(
        gen=dict(seed=3, n_nodes=200000, n_edges=500000, k_min=2, k_max=20, size_exp=2.5, pop_exp=1.2,
                 pop_offset=0.0, dedupe=False),
        burst=dict(burst_rate=1e-4, events_per_burst=50, gap_mean=20.0, span=100_000_000), deltas=[100000])),
}


def run_full(names, threads, timeout):
    """Full-size cases: parallel reference programs only (hours of CPU)."""
    fp = OUT / "full_golden.json"
    for name in names:
        c = FULL_CASES[name]
        if c["kind"] == "static":
            h = static_graph(c["params"])
            counts, wall, _ = rr.run_mochy(h.offsets, h.members, threads=threads, timeout=timeout)
            rec = dict(kind="static", params=c["params"], sha256=digest(h), n_edges=h.n_edges,
                       counts26=counts.tolist(), mochy_par_wall_s=round(wall, 1), threads=threads)
        else:
            h = temporal_graph(c["params"])
            rec = dict(kind="temporal", params=c["params"], sha256=digest(h), n_events=h.n_edges, counts96={},
                       threads=threads)
            for d in c["params"]["deltas"]:
                x, wall, _ = rr.run_thyme(h.offsets, h.members, h.timestamps, d, threads=threads, timeout=timeout)
                rec["counts96"][str(d)] = x.tolist()
                rec[f"thymeP_wall_s_{d}"] = round(wall, 1)
        print(name, "done", flush=True)
        merged = json.loads(fp.read_text()) if fp.exists() else {}  # other runs may have written meanwhile
        merged[name] = rec
        fp.write_text(json.dumps(merged, indent=1))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--timeout", type=float, default=900)
    ap.add_argument("--full", nargs="*", help="run these full-size cases instead")
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args()
    if a.full is not None:
        run_full(a.full or list(FULL_CASES), a.threads, a.timeout)
        return
    sp = OUT / "static_golden.json"
    tp = OUT / "temporal_golden.json"
    sg = json.loads(sp.read_text()) if sp.exists() else {}
    tg = json.loads(tp.read_text()) if tp.exists() else {}
    want = set(a.only) if a.only else None

    dblp = refdata.path("dblp")
    if dblp is not None and (want is None or "dblp" in want):
        off, mem, _ = refdata.read_mochy(dblp)
        c, w, _ = rr.run_mochy(off, mem, threads=None, timeout=a.timeout)
        cp, wp, _ = rr.run_mochy(off, mem, threads=8, timeout=a.timeout)
        assert np.array_equal(c, cp)
        sg["dblp"] = dict(file_sha256=hashlib.sha256(dblp.read_bytes()).hexdigest(), counts26=c.tolist(),
                          n_edges=len(off) - 1, source=refdata.FILES["dblp"], mochy_wall_s=round(w, 3))
        print("dblp", w)

    enron = refdata.path("email-Enron")
    if enron is not None and (want is None or "email-Enron" in want):
        # THyMe's shipped results for this dataset (three exact programs); the
        # data has ties in time, so only tie-independent sums are recorded:
        # the total and the sum per static class of the 96 motifs
        res = {}
        for k in ("thyme", "thymeP", "dp"):
            rp = refdata.path(f"email-Enron-{k}")
            _, c96 = refdata.read_thyme_result(rp)
            res[k] = (int(c96.sum()), refdata.per_static(c96))
        assert res["thyme"] == res["thymeP"] == res["dp"], "shipped results disagree"
        tg["email-Enron"] = dict(file_sha256=refdata.sha256(enron), source=refdata.FILES["email-Enron"],
                                 delta=refdata.ENRON_DELTA, total=res["thymeP"][0], per_static=res["thymeP"][1],
                                 results=[refdata.FILES[f"email-Enron-{k}"] for k in ("thyme", "thymeP", "dp")])
        print("email-Enron", res["thymeP"][0])

    for name, p in STATIC_CASES.items():
        if want is not None and name not in want:
            continue
        h = static_graph(p)
        t0 = time.time()
        c, w, _ = rr.run_mochy(h.offsets, h.members, threads=None, timeout=a.timeout)
        cp, wp, _ = rr.run_mochy(h.offsets, h.members, threads=8, timeout=a.timeout)
        assert np.array_equal(c, cp), name
        sg[name] = dict(params=p, sha256=digest(h), n_edges=h.n_edges, n_members=int(len(h.members)),
                        counts26=c.tolist(), mochy_wall_s=round(w, 3), mochy_par8_wall_s=round(wp, 3))
        print(name, h.n_edges, round(time.time() - t0, 2), "s")
        sp.write_text(json.dumps(sg, indent=1))

    for name, c in TEMPORAL_CASES.items():
        if want is not None and name not in want:
            continue
        h = temporal_graph(c)
        rec = dict(params=c, sha256=digest(h), n_events=h.n_edges, counts96={})
        for d in c["deltas"]:
            t0 = time.time()
            x, w, _ = rr.run_thyme(h.offsets, h.members, h.timestamps, d, threads=None, timeout=a.timeout)
            y, wp, _ = rr.run_thyme(h.offsets, h.members, h.timestamps, d, threads=8, timeout=a.timeout)
            assert np.array_equal(x, y), (name, d)
            rec["counts96"][str(d)] = x.tolist()
            print(name, d, round(time.time() - t0, 2), "s")
        tg[name] = rec
        tp.write_text(json.dumps(tg, indent=1))
    sp.write_text(json.dumps(sg, indent=1))
    tp.write_text(json.dumps(tg, indent=1))


if __name__ == "__main__":
    main()
