"""Benchmark: hyperedge triples classified per second on the 2M-hyperedge
static workload (config 2), plus the update-batch latency of the dynamic
workload when that path is enabled.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
    torchrun --nproc-per-node N bench.py --gpus N ...

A step is one exact static count (all 30 classes, i.e. MoCHy's 26 motifs plus
the four repeated-hyperedge classes) of the resident graph. With N GPUs every
rank holds a replica of the graph and counts one shard of the centres; the
30-class partial counts are summed with one NCCL all-reduce per step, so the
total work is fixed (strong scaling). Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "hyperedge triples classified/sec at 2M edges; update-batch p50/p99 latency"
UNIT = "triples/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--edges", type=int, default=2_000_000)
    ap.add_argument("--nodes", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-traffic", action="store_true")
    ap.add_argument("--write-traffic", default=None,
                    help="compute the algorithmic bytes of this workload live and write them to this JSON file")
    ap.add_argument("--no-tune", action="store_true", help="keep the default closed-phase schedule")
    ap.add_argument("--tune-stride", type=int, default=0,
                    help="autotuner sample: every n-th centre (0: at most 65536 centres)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-sample-edges", type=int, default=40_000,
                    help="the CPU baseline (and the reference arm) counts the first this many hyperedges of the "
                         "workload; the GPU counts the same sample beside it")
    ap.add_argument("--update-batches", type=int, default=100,
                    help="config-3 batches applied to the resident graph after the static steps (0: skip)")
    ap.add_argument("--update-check-every", type=int, default=25,
                    help="full recount checking the running delta sum after every this many batches and after "
                         "the last (0: no check)")
    ap.add_argument("--update-edits", type=int, default=0,
                    help="edits per config-3 batch (0: log-uniform in [1000, 100000], as specified)")
    ap.add_argument("--only", choices=["temporal", "update"], default=None,
                    help="run one section alone on its own workload and print it (for profiling; no headline line)")
    ap.add_argument("--temporal-deltas", default="1000,10000,100000")
    ap.add_argument("--no-temporal", action="store_true")
    ap.add_argument("--no-temporal-cpu", action="store_true")
    ap.add_argument("--temporal-samples", default="1000:50000,10000:10000,100000:1000",
                    help="delta:events pairs: THyMe+ on the first `events` events of config 4 for each delta, "
                         "the GPU on the same sample beside it")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-graphs", type=int, default=256)
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="offered requests per second (Poisson)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="arrival window of the replayed trace")
    ap.add_argument("--serve-low-rate", type=float, default=100.0,
                    help="a second, sustainable offered rate, for latencies that are service times (0: skip)")
    ap.add_argument("--serve-low-seconds", type=float, default=5.0)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    return ap.parse_args()


def laws(args):
    from ipdps26_b200 import workloads

    return workloads.config2_laws(args.edges, args.nodes)


def workload(args):
    from ipdps26_b200 import gen

    p = gen.from_laws(laws(args))
    return p, gen.static(p)


def config_of(args, n_gpus):
    L = laws(args)
    return {
        "workload": "config2-static-count",
        "hyperedges": args.edges,
        "nodes": args.nodes,
        "sizes": "k^-2.2 on [2,100]",
        "popularity": f"Zipf-Mandelbrot s=1.1 q={L.q:g}",
        "seed": 1,
        "parallelism": f"centre-shard x{n_gpus} (replicated store)" if n_gpus > 1 else "single GPU",
        "l2": "inputs larger than L2 (store of tens of GB per step)",
    }


def traffic_key(args):
    return f"config2 seed=1 edges={args.edges} nodes={args.nodes}"


def cached_traffic(args):
    """Algorithmic bytes of the workload, a constant of the seeded input,
    computed once by `bench.py --write-traffic profiles/static_count_bytes.json`."""
    p = ROOT / "profiles" / "static_count_bytes.json"
    if p.exists():
        d = json.loads(p.read_text())
        if d.get("key") == traffic_key(args):
            return d
    return None


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for ln in out.splitlines():
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def mochy_sample(args, path):
    """Writes the first --cpu-sample-edges hyperedges of the workload in
    MoCHy's format with hmgen (host code only; nothing of the engine is
    loaded) and returns the number of hyperedges written."""
    from ipdps26_b200 import workloads

    n, _ = workloads.write_static(laws(args), path, prefix=min(args.cpu_sample_edges, args.edges))
    return n


def run_mochy_sample(path, cores):
    """One timed run of the reference's own OpenMP counter (MoCHy
    main_exact_par, built from the reference sources into oracle/_ref) on all
    host cores: (26 counts, wall seconds including its file parse, its own
    TOTAL_RUNTIME_SECONDS, which leaves the parse out)."""
    from oracle import ref_runner as rr

    return rr.run_mochy_file(path, threads=cores, timeout=3600)


def cpu_baseline(args, h, ctx):
    """MoCHy main_exact_par on the first --cpu-sample-edges hyperedges of the
    workload, timed on the host cores, and the GPU's static count of the very
    same sample beside it: its device time, and whether its 26 counts equal
    the ones MoCHy printed."""
    import tempfile

    from oracle import ref_runner as rr
    from ipdps26_b200 import engine

    if not rr.available("mochy_exact_par"):
        return None
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "sample.txt")
        n = mochy_sample(args, path)
        counts, wall, self_s = run_mochy_sample(path, cores)
    triples = int(counts.sum())
    sub = h.subgraph(n)
    with engine.Graph.from_hypergraph(ctx, sub) as g:
        g.count_static()  # prepares the oriented rows and captures the launches
        ms = []
        for _ in range(5):
            gpu26 = g.count_static()
            ms.append(g.timings().count_ms)
    gpu_s = statistics.median(ms) / 1000.0
    return {"value": triples / wall, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"MoCHy main_exact_par on all {cores} host cores, first {n} hyperedges of the workload "
                      f"(same laws and node universe), {triples} triples (26 motifs) in {wall:.2f} s wall "
                      f"including its file parse ({self_s:.2f} s by its own clock, parse excluded)",
            "sample_hyperedges": n, "wall_s": wall, "self_reported_s": self_s,
            "gpu_same_sample_value": int(gpu26.sum()) / gpu_s, "gpu_same_sample_ms": 1000.0 * gpu_s,
            "gpu_over_cpu_same_sample": (int(gpu26.sum()) / gpu_s) / (triples / wall),
            "parity": bool(np.array_equal(gpu26, counts))}


def pct(xs, q):
    xs = sorted(xs)
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


def update_section(args, g, p, counts30):
    """Config 3: update batches on the resident config-2 graph, each with its
    exact incremental recount (hm_graph_apply_batch with the delta). The
    running sum of the deltas is checked against a full recount after every
    --update-check-every batches and after the last one. Batch sizes are
    log-uniform in [1000, 100000] edits, 80 % insertions drawn from the
    config-2 laws, 20 % deletions uniform over the live hyperedges (seed 2)."""
    from ipdps26_b200 import gen
    from ipdps26_b200._lib import HmError

    rng = np.random.default_rng(2)
    total = counts30.astype(np.int64).copy()
    wall, dev, sizes, checks = [], [], [], []
    every = args.update_check_every
    stopped = None
    for b in range(args.update_batches):
        n_edits = int(np.exp(rng.uniform(np.log(1_000), np.log(100_000))))
        if args.update_edits:
            n_edits = args.update_edits
        live = g.live_ids()
        dels, ins = gen.batch(p, 2_000_000 + b, live, n_edits, 0.8)
        t0 = time.perf_counter()
        try:
            _, delta = g.apply_batch(dels, ins.offsets, ins.members)
        except HmError as err:
            # a batch that fails part-way leaves the store unusable: the
            # section ends here and says where and why
            stopped = {"batch": b + 1, "edits": n_edits, "error": str(err),
                       "device_gb_in_use": g.ctx.memory()[0] / 1e9}
            print(f"[bench] update section stopped: {stopped}", file=sys.stderr, flush=True)
            break
        wall.append(time.perf_counter() - t0)
        dev.append(g.timings().update_ms / 1000.0)
        sizes.append(n_edits)
        total += delta
        if every and ((b + 1) % every == 0 or b + 1 == args.update_batches):
            try:
                full = g.count_static30().astype(np.int64)
            except HmError as err:
                stopped = {"batch": b + 1, "in": "recount check", "error": str(err),
                           "device_gb_in_use": g.ctx.memory()[0] / 1e9}
                print(f"[bench] update section stopped: {stopped}", file=sys.stderr, flush=True)
                break
            checks.append({"after_batch": b + 1, "equal": bool(np.array_equal(full, total)),
                           "recount_ms": round(g.timings().count_ms, 1),
                           "h2h_entries": int(g.info().n_adjacent), "device_gb": g.ctx.memory()[0] / 1e9})
    if not wall:
        return {"batches": 0, "stopped": stopped}
    out = {"batches": len(wall), "stopped": stopped, "edits_min": min(sizes), "edits_max": max(sizes),
           "edits_total": int(sum(sizes)), "p50_ms": 1000 * pct(wall, 50), "p99_ms": 1000 * pct(wall, 99),
           "device_p50_ms": 1000 * pct(dev, 50), "device_p99_ms": 1000 * pct(dev, 99),
           "batches_per_s": len(wall) / sum(wall), "edits_per_s": sum(sizes) / sum(wall),
           "form": "plain per-call (hm_graph_apply_batch with the exact delta)",
           "per_batch_ms": [round(1000 * w, 1) for w in wall], "per_batch_edits": sizes,
           "recount_checks": checks,
           "delta_sum_equals_full_recount": bool(checks) and all(c["equal"] for c in checks)}
    return out


def temporal_samples(args):
    out = []
    for item in args.temporal_samples.split(","):
        d, n = item.split(":")
        out.append((int(d), int(n)))
    return out


def thyme_sample(delta, n_events, cores):
    """THyMe+ (main_thymeP, built from the reference sources into
    oracle/_ref) on the first n_events events of config 4, written in THyMe's
    format by hmgen: (96 counts, wall seconds, its own clock() seconds summed
    over threads)."""
    import tempfile

    from oracle import ref_runner as rr
    from ipdps26_b200 import workloads as W

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "events.txt")
        W.write_temporal(W.CONFIG4, W.CONFIG4_BURSTS, path, prefix=n_events)
        return rr.run_thymeP_file(path, delta, cores, timeout=3600)


def temporal_section(args, ctx):
    """Config 4: THyMe's 96 temporal motifs over 500K bursty events, for
    delta in {1e3, 1e4, 1e5}: device time of one count each, its algorithmic
    bytes (the window-projection walk, hm_graph_temporal_traffic) as a
    roofline, and the reference's own THyMe+ on all host cores on a prefix of
    the same stream with the GPU on that prefix beside it (counts compared)."""
    from oracle import ref_runner as rr
    from ipdps26_b200 import engine, gen

    hbm, peak_kind = peaks()
    h = gen.config4_temporal()
    res = {"events": h.n_edges, "workload": "config4 seed=3 200K nodes, Zipf(1.2), bursty span 1e8",
           "roofline_peak_gbs": hbm, "roofline_peak_kind": peak_kind}
    cores = os.cpu_count() or 1
    with engine.Graph.from_hypergraph(ctx, h) as g:
        for d in (int(x) for x in args.temporal_deltas.split(",")):
            c = g.count_temporal(d)
            ms = []
            for _ in range(3):
                c = g.count_temporal(d)
                ms.append(g.timings().temporal_ms)
            t_ms = statistics.median(ms)
            tr = g.temporal_traffic()
            achieved = tr.b_temp / (t_ms / 1000.0) / 1e9
            res[f"delta_{d}"] = {
                "ms": t_ms, "instances_counted": int(c.sum()),
                "temporal_triples_per_s": float(c.sum()) / (t_ms / 1000.0),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "algorithmic_bytes": int(tr.b_temp),
                             "window_neighbours": int(tr.window_neighbours), "closed_pairs": int(tr.closed_pairs),
                             "open_pairs": int(tr.open_pairs), "kernel": "k_temporal (one block per event)"}}
    if args.no_temporal_cpu or not rr.available("thymeP"):
        return res
    for d, n in temporal_samples(args):
        ref, wall, cpu_s = thyme_sample(d, n, cores)
        sub = h.subgraph(n)
        with engine.Graph.from_hypergraph(ctx, sub) as gs:
            got = gs.count_temporal(d)
            ms = []
            for _ in range(3):
                got = gs.count_temporal(d)
                ms.append(gs.timings().temporal_ms)
        gpu_s = statistics.median(ms) / 1000.0
        inst = int(ref.sum())
        res.setdefault(f"delta_{d}", {})["cpu_baseline"] = {
            "value": inst / wall, "unit": "instances/s", "cores": cores, "kind": "reference",
            "sample": f"THyMe+ main_thymeP on all {cores} host cores, first {n} events of config 4, "
                      f"{inst} instances in {wall:.2f} s wall ({cpu_s:.1f} s of CPU time by its own clock)",
            "sample_events": n, "wall_s": wall, "self_reported_cpu_s": cpu_s,
            "gpu_same_sample_value": float(got.sum()) / gpu_s, "gpu_same_sample_ms": 1000.0 * gpu_s,
            "gpu_over_cpu_same_sample": (float(got.sum()) / gpu_s) / (inst / wall),
            "parity": bool(np.array_equal(got, ref))}
    return res


def serve_section(args, ctx):
    """Config 5: resident graphs behind the request loop. One seeded trace of
    Poisson arrivals (70 % update batches of 100-10,000 edits, 80/20
    insert/delete, 30 % full counts) is replayed at its arrival times through
    four forms:
      per_request          one store per graph, one call per request, every
                           count request a full count (the plain per-call form);
      per_request_kept     the same, counts kept current by the exact deltas
                           after a graph's first full count;
      batched              pooled store, one round of launches serves the
                           oldest waiting request of every graph, kept counts;
      batched_recount      the same, counting in full every time.
    Every result of the four replays must be identical. The batching speed-up
    at equal count semantics is batched / per_request_kept and
    batched_recount / per_request. At --serve-rate both forms are saturated,
    so their latencies are queueing; a second trace at --serve-low-rate, which
    both forms sustain, gives latencies that are service times. Latencies are
    submit-to-done on the server clock."""
    from ipdps26_b200 import engine, gen, serve_trace

    ps = [gen.config5_graph(i) for i in range(args.serve_graphs)]
    hs = [gen.static(p) for p in ps]
    t0 = time.perf_counter()
    trace = serve_trace.make_trace(ps, rate=args.serve_rate, duration=args.serve_seconds, seed=5)
    out = {
        "workload": f"config5: {len(hs)} graphs seeds 100-{99 + len(hs)}, |E| log-uniform [1e3, 2e5], "
                    f"n_nodes=|E|/2, k^-2.5 on [2,25], Zipf-Mandelbrot s=1.2 q={gen.C5_Q:g}; "
                    f"Poisson {args.serve_rate:g} req/s for {args.serve_seconds:g} s (trace seed 5)",
        "hyperedges": int(sum(h.n_edges for h in hs)), "requests": len(trace),
        "update_requests": sum(r.kind == engine.REQ_UPDATE for r in trace),
        "edits": int(sum(r.edits for r in trace if r.kind == engine.REQ_UPDATE)),
        "trace_gen_s": time.perf_counter() - t0, "budget_gb": args.serve_budget_gb,
    }

    def run(name, mode, from_deltas, tr):
        with engine.Server(ctx, mode, mem_budget_bytes=int(args.serve_budget_gb * 1e9),
                           count_from_deltas=from_deltas) as srv:
            for h in hs:
                srv.add_graph(h.offsets, h.members, h.n_nodes)
            t0 = time.perf_counter()
            srv.start()
            build_s = time.perf_counter() - t0
            rep = serve_trace.replay(srv, tr)
            st = srv.stats()
        return rep, {**serve_trace.summarize(tr, rep), "build_s": build_s, "rounds": int(st.rounds),
                     "device_gb_after": st.device_bytes / 1e9}

    forms = (("per_request", engine.SERVE_PER_REQUEST, False), ("per_request_kept", engine.SERVE_PER_REQUEST, True),
             ("batched", engine.SERVE_BATCHED, True), ("batched_recount", engine.SERVE_BATCHED, False))
    reps = {}
    for name, mode, from_deltas in forms:
        reps[name], out[name] = run(name, mode, from_deltas, trace)
    base = reps["per_request"]
    out["same_results"] = all(serve_trace.same_results(base, reps[k]) for k in reps if k != "per_request")
    ups = {k: out[k]["update_batches_per_s"] for k, _, _ in forms}
    out["update_throughput_ratio"] = ups["batched"] / ups["per_request"]
    out["batching_ratio_kept_counts"] = ups["batched"] / ups["per_request_kept"]
    out["batching_only_ratio"] = ups["batched_recount"] / ups["per_request"]
    if args.serve_low_rate > 0:
        low = serve_trace.make_trace(ps, rate=args.serve_low_rate, duration=args.serve_low_seconds, seed=6)
        lo = {"offered_req_per_s": args.serve_low_rate, "seconds": args.serve_low_seconds, "requests": len(low)}
        lreps = {}
        for name, mode, from_deltas in (forms[1], forms[2]):
            lreps[name], lo[name] = run(name, mode, from_deltas, low)
        lo["same_results"] = serve_trace.same_results(lreps["per_request_kept"], lreps["batched"])
        out["sustained"] = lo
    return out


def reference_arm(args, rank, world):
    """The reference's own CPU counter (MoCHy main_exact_par on all host
    cores, from oracle/_ref) on a bounded sample of the workload: its first
    --cpu-sample-edges hyperedges, written by the host-only hmgen tool, so
    that this process maps nothing of the engine. Each step is one run of the
    program on that sample (wall time including its file parse). The sample is
    stated in `config`: the reference cannot count the full 2M-hyperedge
    workload in a bench run (days of CPU time at its measured rate)."""
    if rank != 0:
        return
    import tempfile

    from oracle import ref_runner as rr

    if not rr.available("mochy_exact_par"):
        print(json.dumps({"impl": "reference", "unavailable": "reference counter (oracle/_ref) not built here"}))
        return
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "sample.txt")
        n = mochy_sample(args, path)
        for _ in range(args.warmup):
            run_mochy_sample(path, cores)
        walls, selfs, triples = [], [], 0
        for _ in range(args.steps):
            c, w, s_self = run_mochy_sample(path, cores)
            walls.append(w)
            selfs.append(s_self)
            triples = int(c.sum())
    t = sum(walls)
    value = triples * args.steps / t
    cfg = {**config_of(args, 1), "parallelism": f"OpenMP, {cores} host threads",
           "sample_hyperedges": n,
           "sample": f"first {n} of the {args.edges} hyperedges (same laws and node universe)"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "int64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"MoCHy main_exact_par, first {n} hyperedges of the workload, {triples} triples "
                                   f"(26 motifs) per run, {t / args.steps:.2f} s wall per run including its file "
                                   f"parse ({statistics.mean(selfs):.2f} s by its own clock)",
                         "sample_hyperedges": n},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def engine_arm(args, rank, world, local_rank):
    import torch

    from ipdps26_b200 import engine, shard

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    p, h = workload(args)
    ctx = engine.Context(local_rank)
    g = engine.Graph.from_hypergraph(ctx, h)
    stream = torch.cuda.ExternalStream(engine.lib.hm_ctx_stream(ctx.handle))

    # the launch schedule, picked by the autotuner on rank 0 before any timing;
    # every rank must split the work list the same way for the shards to add up
    tune = None
    if not args.no_tune:
        if rank == 0:
            tune = g.autotune(args.tune_stride).as_dict()
        if world > 1:
            g.set_schedule(*shard.agree_schedule(g.schedule, dist, f"cuda:{local_rank}"))

    def step():
        part = g.count_static30_shard(rank, world)
        if world > 1:
            part = shard.allreduce_counts(part, dist, f"cuda:{local_rank}")
        return part

    for _ in range(args.warmup):
        counts = step()
    closed_ms, open_ms = [], []
    with ClockSampler(local_rank) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            counts = step()
            t = g.timings()
            closed_ms.append(t.closed_ms)
            open_ms.append(t.open_ms)
        e1.record(stream)
        torch.cuda.synchronize()
        closed_tri = int(g.timings().closed_triangles)
        wall = time.perf_counter() - t0
        if world > 1:
            dist.barrier()
    dev_s = e0.elapsed_time(e1) / 1000.0
    if world > 1:
        dev_s = shard.max_over_ranks(dev_s, dist, f"cuda:{local_rank}")
        # each rank enumerated the closed triangles of its own shard
        closed_tri = int(shard.allreduce_counts(np.array([closed_tri], np.uint64), dist, f"cuda:{local_rank}")[0])
    triples = int(counts.astype(np.uint64).sum())
    value = triples * args.steps / dev_s

    result = None
    if rank == 0:
        hbm, peak_kind = peaks()
        info = g.info()
        roof = None
        if not args.no_traffic:
            tr = cached_traffic(args)
            if tr is None:
                t = g.traffic()
                tr = {"b_static": t.b_static, "store_bytes": t.store_bytes, "merge_bytes": t.merge_bytes,
                      "closed_pair_bytes": t.closed_pair_bytes, "kernel_bytes": t.kernel_bytes, "probes": t.probes,
                      "key": traffic_key(args)}
                if args.write_traffic:
                    Path(args.write_traffic).write_text(json.dumps(tr, indent=1))
            # one step = the count kernels; per-launch duration from CUDA events
            t_launch = (statistics.mean(closed_ms) + statistics.mean(open_ms)) / 1000.0
            achieved = tr["b_static"] / t_launch / 1e9
            traffic = None
            tp = ROOT / "profiles" / "static_count_dram.json"
            if tp.exists():
                tj = json.loads(tp.read_text())
                if tj.get("key") == traffic_key(args):
                    traffic = tj.get("dram_bytes_per_step")
            roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "traffic": traffic, "peak_kind": peak_kind,
                    "traffic_gbs": traffic / t_launch / 1e9 if traffic else None,
                    "algorithmic_bytes": tr["b_static"], "kernel_model_bytes": tr["kernel_bytes"],
                    "kernel_model_gbs": tr["kernel_bytes"] / t_launch / 1e9,
                    "kernel": "k_open_pairs + k_closed (three launch shapes split by the tuned schedule, "
                              "replayed as two captured CUDA graphs): one static count",
                    "basis": "achieved = algorithmic_bytes (the reference algorithm's merge bytes per count) "
                             "/ count time; the kernel probes hashed rows instead and moves `traffic` bytes "
                             "(ncu), so frac can pass 1",
                    "closed_ms": statistics.mean(closed_ms), "open_ms": statistics.mean(open_ms)}
        e2e = None
        if not args.no_e2e:
            # through the public API from host buffers: build (H2D of the CSR),
            # count, read the 26 counts back; pinned host copies of the inputs
            off = torch.from_numpy(h.offsets.view(np.int64)).pin_memory().numpy().view(np.uint64)
            mem = torch.from_numpy(h.members.view(np.int32)).pin_memory().numpy().view(np.uint32)
            times = []
            for _ in range(args.e2e_steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                with engine.Graph(ctx, off, mem, h.n_nodes) as g2:
                    g2.set_schedule(*g.schedule)  # the tuned schedule of this workload
                    c26 = g2.count_static()
                times.append(time.perf_counter() - t0)
            e2e = {"value": int(c26.sum()) / statistics.mean(times), "unit": UNIT,
                   "h2d_bytes_per_step": int(off.nbytes + mem.nbytes), "d2h_bytes_per_step": 26 * 8,
                   "s_per_step": statistics.mean(times),
                   "note": "26 reported motifs; build of H2V/V2H/H2H included"}
        mem_gb = {"after_static_and_e2e": ctx.memory()[0] / 1e9}
        base = None
        if world == 1 and not args.no_cpu_baseline:
            base = cpu_baseline(args, h, ctx)
        mem_gb["before_updates"] = ctx.memory()[0] / 1e9
        print(f"[bench] device memory in use: {mem_gb}", file=sys.stderr, flush=True)
        updates = None
        if args.update_batches > 0:
            updates = update_section(args, g, p, counts)
        g_sched = g.schedule
        g.close()  # the sections below build their own stores
        temporal = None
        if not args.no_temporal:
            temporal = temporal_section(args, ctx)
        serve = None
        if not args.no_serve:
            serve = serve_section(args, ctx)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            # per step: k_open_pairs and the three closed-phase launch shapes
            "config": {**config_of(args, world), "schedule": list(g_sched)}, "gpu_launches": 4 * args.steps,
            "autotune": tune,
            "triples_per_step": triples, "closed_triangles_per_step": closed_tri,
            "closed_triangles_per_s": closed_tri * args.steps / dev_s,
            "wall_s": wall, "clocks": clk.summary(), "roofline": roof, "e2e": e2e, "cpu_baseline": base,
            "graph": {"h2h_entries": int(info.n_adjacent), "oriented_entries": int(info.n_oriented),
                      "device_gb": info.device_bytes / 1e9},
            "update_batches": updates, "temporal": temporal, "served": serve, "device_memory_gb": mem_gb,
        }
        print(json.dumps(result), flush=True)
    g.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def section_only(args):
    """One section on its own workload (for profiling one kernel family with
    committed code): --only temporal (config 4 at --temporal-deltas) or
    --only update (--update-batches of --update-edits on the workload at
    --edges / --nodes)."""
    from ipdps26_b200 import engine

    with engine.Context(0) as ctx:
        if args.only == "temporal":
            out = temporal_section(args, ctx)
        else:
            p, h = workload(args)
            with engine.Graph.from_hypergraph(ctx, h) as g:
                out = update_section(args, g, p, g.count_static30())
    print(json.dumps({"section": args.only, **out}), flush=True)


def main():
    args = parse()
    if args.only:
        section_only(args)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if "RANK" not in os.environ:
        world = 1 if args.gpus == 1 else args.gpus
        if world != 1:
            raise SystemExit("for --gpus > 1 launch with torchrun (one process per GPU)")
    if args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        engine_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
