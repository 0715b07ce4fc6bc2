"""Python view of the engine's C ABI (include/hmotif.h).

Mirrors the reference's host interface for this path: a store built once
from hyperedge lists (constructCBST / CBSTOperations::construct,
dynamicHyperGraph/include/structure.hpp:38-64), batch insert/delete, query,
and count calls returning MoCHy's 26 static and THyMe's 96 temporal h-motif
counts. Every call goes through libhmotif.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _lib
from ._lib import check, lib, ptr, u32p, u64p, i64p, vp

N_STATIC_CLASSES = 30
N_STATIC_MOTIFS = 26
N_TEMPORAL_MOTIFS = 96


class GraphInfo(C.Structure):
    _fields_ = [
        ("n_slots", C.c_uint32),
        ("n_live", C.c_uint32),
        ("n_nodes", C.c_uint32),
        ("temporal", C.c_int32),
        ("n_members", C.c_uint64),
        ("n_adjacent", C.c_uint64),
        ("n_oriented", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]


class Traffic(C.Structure):
    _fields_ = [
        ("store_bytes", C.c_uint64),
        ("merge_bytes", C.c_uint64),
        ("closed_pair_bytes", C.c_uint64),
        ("b_static", C.c_uint64),
        ("probes", C.c_uint64),
        ("kernel_bytes", C.c_uint64),
        ("closed_triangles", C.c_uint64),
    ]


class Timings(C.Structure):
    _fields_ = [
        ("open_ms", C.c_float),
        ("closed_ms", C.c_float),
        ("count_ms", C.c_float),
        ("update_ms", C.c_float),
        ("temporal_ms", C.c_float),
        ("closed_triangles", C.c_uint64),
    ]


class TemporalTraffic(C.Structure):
    _fields_ = [
        ("events", C.c_uint64),
        ("delta", C.c_int64),
        ("window_neighbours", C.c_uint64),
        ("closed_pairs", C.c_uint64),
        ("open_pairs", C.c_uint64),
        ("b_temp", C.c_uint64),
    ]


class Schedule(C.Structure):
    """Launch splits of the static and touched-triple counts (hm_schedule)."""

    _fields_ = [
        ("warp_row", C.c_uint32),
        ("small_row", C.c_uint32),
        ("touch_warp_row", C.c_uint32),
        ("touch_mid_row", C.c_uint32),
    ]

    def astuple(self) -> tuple[int, int, int, int]:
        return (self.warp_row, self.small_row, self.touch_warp_row, self.touch_mid_row)


TUNE_MAX_CANDIDATES = 16


class TuneReport(C.Structure):
    _fields_ = [
        ("n_candidates", C.c_uint32),
        ("best", C.c_uint32),
        ("sample_stride", C.c_uint32),
        ("sampled", C.c_uint32),
        ("rows", (C.c_uint32 * 2) * TUNE_MAX_CANDIDATES),
        ("ms", C.c_float * TUNE_MAX_CANDIDATES),
        ("touch_n_candidates", C.c_uint32),
        ("touch_best", C.c_uint32),
        ("touch_sampled", C.c_uint32),
        ("touch_rows", (C.c_uint32 * 2) * TUNE_MAX_CANDIDATES),
        ("touch_ms", C.c_float * TUNE_MAX_CANDIDATES),
        ("tune_ms", C.c_float),
    ]

    def as_dict(self) -> dict:
        def part(rows, ms, n, best):
            return {"best": list(rows[best]), "default": list(rows[0]),
                    "candidates": [[*rows[i], round(float(ms[i]), 3)] for i in range(n)]}

        return {
            "static": {**part(self.rows, self.ms, self.n_candidates, self.best),
                       "sample_stride": self.sample_stride, "sampled_centres": self.sampled,
                       "ms": "closed-phase device time of the sample"},
            "touch": {**part(self.touch_rows, self.touch_ms, self.touch_n_candidates, self.touch_best),
                      "sampled_rows": self.touch_sampled, "ms": "wall time of the sample's touched-triple count"},
            "tune_ms": round(float(self.tune_ms), 1),
        }


class ServeConfig(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("max_batch_requests", C.c_uint32),
        ("max_batch_edits", C.c_uint64),
        ("mem_budget_bytes", C.c_size_t),
        ("count_from_deltas", C.c_int32),
        ("pad_", C.c_int32),
    ]


class ServeResult(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("graph", C.c_uint32),
        ("kind", C.c_int32),
        ("status", C.c_int32),
        ("n_assigned", C.c_uint32),
        ("delta30", C.c_int64 * 30),
        ("counts30", C.c_uint64 * 30),
        ("submit_ms", C.c_double),
        ("start_ms", C.c_double),
        ("done_ms", C.c_double),
        ("round_requests", C.c_uint32),
        ("pad_", C.c_uint32),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("rounds", C.c_uint64),
        ("requests_done", C.c_uint64),
        ("requests_failed", C.c_uint64),
        ("edits_done", C.c_uint64),
        ("waiting", C.c_uint64),
        ("deferred_budget", C.c_uint64),
        ("busy_ms", C.c_double),
        ("device_bytes", C.c_size_t),
    ]


_lib.bind(
    {
        "hm_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(vp)]),
        "hm_ctx_destroy": (C.c_int, [vp]),
        "hm_ctx_memory": (C.c_int, [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
        "hm_ctx_stream": (vp, [vp]),
        "hm_debug_fail_allocations_after": (C.c_int, [C.c_longlong]),
        "hm_graph_build": (C.c_int, [vp, u64p, u32p, C.c_uint32, C.c_uint32, i64p, C.POINTER(vp)]),
        "hm_graph_destroy": (C.c_int, [vp]),
        "hm_graph_info": (C.c_int, [vp, C.POINTER(GraphInfo)]),
        "hm_graph_query": (C.c_int, [vp, u32p, C.c_uint32, u64p, u32p, C.c_size_t]),
        "hm_graph_timings": (C.c_int, [vp, C.POINTER(Timings)]),
        "hm_count_static": (C.c_int, [vp, u64p]),
        "hm_count_static30": (C.c_int, [vp, u64p]),
        "hm_count_static30_shard": (C.c_int, [vp, C.c_uint32, C.c_uint32, u64p]),
        "hm_count_static30_async": (C.c_int, [vp, vp, vp]),
        "hm_graph_traffic": (C.c_int, [vp, C.POINTER(Traffic)]),
        "hm_graph_apply_batch": (C.c_int, [vp, u32p, C.c_uint32, u64p, u32p, C.c_uint32, u32p, i64p]),
        "hm_graph_live_ids": (C.c_int, [vp, u32p, C.c_uint32, C.POINTER(C.c_uint32)]),
        "hm_count_touching30": (C.c_int, [vp, u32p, C.c_uint32, u64p]),
        "hm_count_temporal": (C.c_int, [vp, C.c_int64, u64p]),
        "hm_graph_temporal_traffic": (C.c_int, [vp, C.POINTER(TemporalTraffic)]),
        "hm_count_temporal_async": (C.c_int, [vp, C.c_int64, vp, vp]),
        "hm_graph_apply_batch_async": (C.c_int, [vp, u32p, C.c_uint32, u64p, u32p, C.c_uint32, u32p, vp, vp]),
        "hm_graph_fill": (C.c_int, [vp, u32p, C.c_uint32, u32p, u64p, i64p]),
        "hm_graph_unfill": (C.c_int, [vp, u32p, C.c_uint32, u32p, u64p, i64p]),
        "hm_debug_touch_orientation": (C.c_int, [vp, C.c_int]),
        "hm_debug_static_groups": (C.c_int, [vp, C.c_int]),
        "hm_count_vertex_triads": (C.c_int, [vp, u64p]),
        "hm_graph_set_schedule": (C.c_int, [vp, C.POINTER(Schedule)]),
        "hm_graph_get_schedule": (C.c_int, [vp, C.POINTER(Schedule)]),
        "hm_graph_autotune": (C.c_int, [vp, C.c_uint32, C.POINTER(TuneReport)]),
        "hm_serve_create": (C.c_int, [vp, C.POINTER(ServeConfig), C.POINTER(vp)]),
        "hm_serve_add_graph": (C.c_int, [vp, u64p, u32p, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]),
        "hm_serve_start": (C.c_int, [vp]),
        "hm_serve_submit_update": (C.c_int, [vp, C.c_uint32, u32p, C.c_uint32, u64p, u32p, C.c_uint32,
                                             C.POINTER(C.c_uint64)]),
        "hm_serve_submit_count": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_uint64)]),
        "hm_serve_wait": (C.c_int, [vp, C.c_uint64, C.POINTER(ServeResult), u32p, C.c_uint32]),
        "hm_serve_drain": (C.c_int, [vp]),
        "hm_serve_stats": (C.c_int, [vp, C.POINTER(ServeStats)]),
        "hm_serve_live_ids": (C.c_int, [vp, C.c_uint32, u32p, C.c_uint32, C.POINTER(C.c_uint32)]),
        "hm_serve_destroy": (C.c_int, [vp]),
        "hm_window_create": (C.c_int, [vp, C.c_uint32, C.POINTER(vp)]),
        "hm_window_destroy": (C.c_int, [vp]),
        "hm_window_set_layer": (C.c_int, [vp, C.c_int, u64p, u32p, C.c_uint32]),
        "hm_window_rotate": (C.c_int, [vp]),
        "hm_window_reset_layer": (C.c_int, [vp, C.c_int]),
        "hm_window_fill": (C.c_int, [vp, C.c_int, u32p, C.c_uint32, u32p, u64p]),
        "hm_window_unfill": (C.c_int, [vp, C.c_int, u32p, C.c_uint32, u32p, u64p]),
        "hm_window_apply_deltas_file": (C.c_int, [vp, C.c_char_p]),
        "hm_window_layer_size": (C.c_int, [vp, C.c_int, C.POINTER(C.c_uint32)]),
        "hm_window_count30": (C.c_int, [vp, u64p]),
        "hm_classify_static": (C.c_int, [C.c_int]),
        "hm_classify_temporal": (C.c_int, [C.c_int]),
    }
)


class Context:
    """One CUDA device, one stream, one device-memory budget."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0):
        h = vp()
        check(lib.hm_ctx_create(device, mem_budget_bytes, C.byref(h)), "hm_ctx_create")
        self._h = h
        self.device = device
        self._children = weakref.WeakSet()  # graphs are released before the context

    @property
    def handle(self):
        return self._h

    def memory(self) -> tuple[int, int]:
        used, budget = C.c_size_t(), C.c_size_t()
        check(lib.hm_ctx_memory(self._h, C.byref(used), C.byref(budget)), "hm_ctx_memory")
        return used.value, budget.value

    def close(self) -> None:
        if self._h:
            for child in list(self._children):
                child.close()
            lib.hm_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _csr_arrays(offsets, members):
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    mem = np.ascontiguousarray(members, dtype=np.uint32)
    return off, mem


class Graph:
    """A device-resident hypergraph (H2V, V2H, H2H) owned by a Context."""

    def __init__(self, ctx: Context, offsets, members, n_nodes: int, timestamps=None):
        off, mem = _csr_arrays(offsets, members)
        ts = None if timestamps is None else np.ascontiguousarray(timestamps, dtype=np.int64)
        n_edges = len(off) - 1
        h = vp()
        check(
            lib.hm_graph_build(ctx.handle, ptr(off, C.c_uint64), ptr(mem, C.c_uint32), n_edges, int(n_nodes),
                               ptr(ts, C.c_int64), C.byref(h)),
            "hm_graph_build",
        )
        self._h = h
        self.ctx = ctx
        ctx._children.add(self)

    @classmethod
    def from_hypergraph(cls, ctx: Context, hg) -> "Graph":
        return cls(ctx, hg.offsets, hg.members, hg.n_nodes, hg.timestamps)

    @property
    def handle(self):
        return self._h

    def info(self) -> GraphInfo:
        i = GraphInfo()
        check(lib.hm_graph_info(self._h, C.byref(i)), "hm_graph_info")
        return i

    def timings(self) -> Timings:
        t = Timings()
        check(lib.hm_graph_timings(self._h, C.byref(t)), "hm_graph_timings")
        return t

    def count_static(self) -> np.ndarray:
        out = np.zeros(N_STATIC_MOTIFS, np.uint64)
        check(lib.hm_count_static(self._h, ptr(out, C.c_uint64)), "hm_count_static")
        return out

    def count_static30(self) -> np.ndarray:
        out = np.zeros(N_STATIC_CLASSES, np.uint64)
        check(lib.hm_count_static30(self._h, ptr(out, C.c_uint64)), "hm_count_static30")
        return out

    def count_static30_shard(self, shard: int, n_shards: int) -> np.ndarray:
        out = np.zeros(N_STATIC_CLASSES, np.uint64)
        check(lib.hm_count_static30_shard(self._h, shard, n_shards, ptr(out, C.c_uint64)), "hm_count_static30_shard")
        return out

    def count_static30_async(self, d_out30: int, stream: int | None = None) -> None:
        """Queues the 30-class count after the work on `stream` (a
        cudaStream_t as an int, 0 being the legacy default stream that torch's
        default stream is; None: the context stream); the counts land in the
        30 uint64 at device address d_out30 without a host wait."""
        s = lib.hm_ctx_stream(self.ctx.handle) if stream is None else stream
        check(lib.hm_count_static30_async(self._h, vp(d_out30), vp(s)), "hm_count_static30_async")

    def traffic(self) -> Traffic:
        t = Traffic()
        check(lib.hm_graph_traffic(self._h, C.byref(t)), "hm_graph_traffic")
        return t

    def apply_batch(self, del_ids, ins_offsets=None, ins_members=None, delta: bool = True):
        """Delete then insert; returns (assigned ids, 30-class delta or None)."""
        d = np.ascontiguousarray(del_ids if del_ids is not None else [], dtype=np.uint32)
        if ins_offsets is None:
            ins_offsets, ins_members = np.zeros(1, np.uint64), np.zeros(0, np.uint32)
        off, mem = _csr_arrays(ins_offsets, ins_members)
        n_ins = len(off) - 1
        ids = np.zeros(max(n_ins, 1), np.uint32)
        dl = np.zeros(N_STATIC_CLASSES, np.int64) if delta else None
        check(lib.hm_graph_apply_batch(self._h, ptr(d, C.c_uint32), len(d), ptr(off, C.c_uint64),
                                       ptr(mem if len(mem) else np.zeros(1, np.uint32), C.c_uint32), n_ins,
                                       ptr(ids, C.c_uint32), ptr(dl, C.c_int64)), "hm_graph_apply_batch")
        return ids[:n_ins].copy(), dl

    def apply_batch_async(self, del_ids, ins_offsets=None, ins_members=None, d_delta30: int | None = None,
                          stream: int | None = None) -> np.ndarray:
        """hm_graph_apply_batch ordered on `stream` (a cudaStream_t as an int,
        0 the legacy default stream; None the context stream); the delta, if
        d_delta30 is a device address, lands there. Returns the assigned ids."""
        d = np.ascontiguousarray(del_ids if del_ids is not None else [], dtype=np.uint32)
        if ins_offsets is None:
            ins_offsets, ins_members = np.zeros(1, np.uint64), np.zeros(0, np.uint32)
        off, mem = _csr_arrays(ins_offsets, ins_members)
        n_ins = len(off) - 1
        ids = np.zeros(max(n_ins, 1), np.uint32)
        s = lib.hm_ctx_stream(self.ctx.handle) if stream is None else stream
        check(lib.hm_graph_apply_batch_async(self._h, ptr(d, C.c_uint32), len(d), ptr(off, C.c_uint64),
                                             ptr(mem if len(mem) else np.zeros(1, np.uint32), C.c_uint32), n_ins,
                                             ptr(ids, C.c_uint32), vp(d_delta30) if d_delta30 else None, vp(s)),
              "hm_graph_apply_batch_async")
        return ids[:n_ins].copy()

    def _members_edit(self, fn, name, ids, values_per_id):
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        vals = [np.asarray(v, dtype=np.uint32) for v in values_per_id]
        if len(vals) != len(ids):
            raise ValueError(f"{name}: one value list per id")
        prefix = np.cumsum([len(v) for v in vals]).astype(np.uint64) if len(vals) else np.zeros(0, np.uint64)
        flat = np.concatenate(vals) if vals and sum(map(len, vals)) else np.zeros(1, np.uint32)
        dl = np.zeros(N_STATIC_CLASSES, np.int64)
        check(fn(self._h, ptr(ids, C.c_uint32), len(ids), ptr(flat, C.c_uint32),
                 ptr(prefix if len(prefix) else np.zeros(1, np.uint64), C.c_uint64), ptr(dl, C.c_int64)), name)
        return dl

    def fill(self, ids, values_per_id) -> np.ndarray:
        """Keyed fill (fillCBST): adds values_per_id[i] to the members of live
        hyperedge ids[i], ids kept; returns the exact 30-class delta."""
        return self._members_edit(lib.hm_graph_fill, "hm_graph_fill", ids, values_per_id)

    def unfill(self, ids, values_per_id) -> np.ndarray:
        """Keyed unfill (unfillCBST): removes the values from the members."""
        return self._members_edit(lib.hm_graph_unfill, "hm_graph_unfill", ids, values_per_id)

    def live_ids(self) -> np.ndarray:
        n = C.c_uint32()
        check(lib.hm_graph_live_ids(self._h, None, 0, C.byref(n)), "hm_graph_live_ids")
        out = np.zeros(max(n.value, 1), np.uint32)
        check(lib.hm_graph_live_ids(self._h, ptr(out, C.c_uint32), len(out), C.byref(n)), "hm_graph_live_ids")
        return out[: n.value].copy()

    def count_temporal(self, delta: int) -> np.ndarray:
        out = np.zeros(N_TEMPORAL_MOTIFS, np.uint64)
        check(lib.hm_count_temporal(self._h, int(delta), ptr(out, C.c_uint64)), "hm_count_temporal")
        return out

    def count_temporal_async(self, delta: int, d_out96: int, stream: int | None = None) -> None:
        """Queues the 96-motif count after the work on `stream` (0: the legacy
        default stream; None: the context stream) into device memory d_out96."""
        s = lib.hm_ctx_stream(self.ctx.handle) if stream is None else stream
        check(lib.hm_count_temporal_async(self._h, int(delta), vp(d_out96), vp(s)), "hm_count_temporal_async")

    def temporal_traffic(self) -> TemporalTraffic:
        """Window-projection sizes and algorithmic bytes of the last temporal count."""
        t = TemporalTraffic()
        check(lib.hm_graph_temporal_traffic(self._h, C.byref(t)), "hm_graph_temporal_traffic")
        return t

    def count_touching30(self, ids) -> np.ndarray:
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        out = np.zeros(N_STATIC_CLASSES, np.uint64)
        check(lib.hm_count_touching30(self._h, ptr(ids, C.c_uint32), len(ids), ptr(out, C.c_uint64)),
              "hm_count_touching30")
        return out

    def count_vertex_triads(self) -> np.ndarray:
        """The reference's type 1, 2 and 3 vertex-triad counts."""
        out = np.zeros(3, np.uint64)
        check(lib.hm_count_vertex_triads(self._h, ptr(out, C.c_uint64)), "hm_count_vertex_triads")
        return out

    @property
    def schedule(self) -> tuple[int, int, int, int]:
        """(warp_row, small_row, touch_warp_row, touch_mid_row): the launch
        splits of the static and touched-triple counts."""
        sc = Schedule()
        check(lib.hm_graph_get_schedule(self._h, C.byref(sc)), "hm_graph_get_schedule")
        return sc.astuple()

    def set_schedule(self, warp_row: int, small_row: int, touch_warp_row: int | None = None,
                     touch_mid_row: int | None = None) -> None:
        """Sets the static split; the touched-triple split too when given."""
        cur = self.schedule
        sc = Schedule(warp_row, small_row, cur[2] if touch_warp_row is None else touch_warp_row,
                      cur[3] if touch_mid_row is None else touch_mid_row)
        check(lib.hm_graph_set_schedule(self._h, C.byref(sc)), "hm_graph_set_schedule")

    def autotune(self, sample_stride: int = 0) -> TuneReport:
        """Times the candidate schedules on a sample of the centres and keeps
        the fastest (hm_graph_autotune)."""
        r = TuneReport()
        check(lib.hm_graph_autotune(self._h, int(sample_stride), C.byref(r)), "hm_graph_autotune")
        return r

    def set_static_groups(self, on: bool) -> None:
        """Walk of the static count: grouped rows with the shared-member group
        counted in bulk (default), or every oriented entry (same counts)."""
        check(lib.hm_debug_static_groups(self._h, int(on)), "hm_debug_static_groups")

    def set_touch_orientation(self, by_id: bool) -> None:
        """Walk order of the touched-triple counts (same counts either way)."""
        check(lib.hm_debug_touch_orientation(self._h, int(by_id)), "hm_debug_touch_orientation")

    def query(self, ids) -> list[np.ndarray]:
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        n = len(ids)
        off = np.zeros(n + 1, np.uint64)
        cap = 256 * max(n, 1)
        mem = np.zeros(cap, np.uint32)
        check(lib.hm_graph_query(self._h, ptr(ids, C.c_uint32), n, ptr(off, C.c_uint64), ptr(mem, C.c_uint32), cap),
              "hm_graph_query")
        return [mem[off[i] : off[i + 1]].copy() for i in range(n)]

    def close(self) -> None:
        if self._h:
            lib.hm_graph_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


OLDER, MIDDLE, NEWEST = 0, 1, 2


class Window:
    """Three-layer temporal window (Older, Middle, Newest) and its strictly
    increasing 30-class count (hm_window_* in hmotif.h)."""

    def __init__(self, ctx: Context, n_nodes: int):
        h = vp()
        check(lib.hm_window_create(ctx.handle, int(n_nodes), C.byref(h)), "hm_window_create")
        self._h = h
        self.ctx = ctx
        ctx._children.add(self)

    def set_layer(self, layer: int, offsets, members) -> None:
        off, mem = _csr_arrays(offsets, members)
        check(lib.hm_window_set_layer(self._h, layer, ptr(off, C.c_uint64),
                                      ptr(mem if len(mem) else np.zeros(1, np.uint32), C.c_uint32), len(off) - 1),
              "hm_window_set_layer")

    def rotate(self) -> None:
        check(lib.hm_window_rotate(self._h), "hm_window_rotate")

    def reset_layer(self, layer: int) -> None:
        check(lib.hm_window_reset_layer(self._h, layer), "hm_window_reset_layer")

    def _fill(self, fn, name, layer, ids, values_per_id):
        ids = np.ascontiguousarray(ids, np.uint32)
        vals = np.ascontiguousarray(np.concatenate([np.asarray(v, np.uint32) for v in values_per_id])
                                    if len(values_per_id) else np.zeros(0, np.uint32), np.uint32)
        pre = np.cumsum([len(v) for v in values_per_id]).astype(np.uint64) if len(values_per_id) else np.zeros(0, np.uint64)
        check(fn(self._h, layer, ptr(ids if len(ids) else np.zeros(1, np.uint32), C.c_uint32), len(ids),
                 ptr(vals if len(vals) else np.zeros(1, np.uint32), C.c_uint32),
                 ptr(pre if len(pre) else np.zeros(1, np.uint64), C.c_uint64)), name)

    def fill(self, layer: int, ids, values_per_id) -> None:
        self._fill(lib.hm_window_fill, "hm_window_fill", layer, ids, values_per_id)

    def unfill(self, layer: int, ids, values_per_id) -> None:
        self._fill(lib.hm_window_unfill, "hm_window_unfill", layer, ids, values_per_id)

    def apply_deltas_file(self, path) -> None:
        check(lib.hm_window_apply_deltas_file(self._h, str(path).encode()), "hm_window_apply_deltas_file")

    def layer_size(self, layer: int) -> int:
        n = C.c_uint32()
        check(lib.hm_window_layer_size(self._h, layer, C.byref(n)), "hm_window_layer_size")
        return n.value

    def count30(self) -> np.ndarray:
        out = np.zeros(N_STATIC_CLASSES, np.uint64)
        check(lib.hm_window_count30(self._h, ptr(out, C.c_uint64)), "hm_window_count30")
        return out

    def close(self) -> None:
        if self._h:
            lib.hm_window_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SERVE_BATCHED = 0
SERVE_PER_REQUEST = 1
REQ_UPDATE = 0
REQ_COUNT = 1


class Server:
    """Many resident graphs behind one request loop (hm_serve_* in hmotif.h).

    ``mode`` SERVE_BATCHED serves one request of every waiting graph per
    round over a pooled store; SERVE_PER_REQUEST serves them one call at a
    time on per-graph stores. With ``count_from_deltas`` a graph's counts,
    once counted in full, are kept current by the exact deltas of its
    updates and answer its later count requests. Results are the same in
    every form.
    """

    def __init__(self, ctx: Context, mode: int = SERVE_BATCHED, max_batch_requests: int = 0,
                 max_batch_edits: int = 0, mem_budget_bytes: int = 0, count_from_deltas: bool = False):
        cfg = ServeConfig(mode, max_batch_requests, max_batch_edits, mem_budget_bytes, int(count_from_deltas))
        h = vp()
        check(lib.hm_serve_create(ctx.handle, C.byref(cfg), C.byref(h)), "hm_serve_create")
        self._h = h
        self.ctx = ctx
        self.mode = mode
        ctx._children.add(self)

    def add_graph(self, offsets, members, n_nodes: int) -> int:
        off, mem = _csr_arrays(offsets, members)
        gid = C.c_uint32()
        check(lib.hm_serve_add_graph(self._h, ptr(off, C.c_uint64),
                                     ptr(mem if len(mem) else np.zeros(1, np.uint32), C.c_uint32), len(off) - 1,
                                     int(n_nodes), C.byref(gid)), "hm_serve_add_graph")
        return gid.value

    def start(self) -> None:
        check(lib.hm_serve_start(self._h), "hm_serve_start")

    def submit_update(self, graph: int, del_ids=None, ins_offsets=None, ins_members=None) -> int:
        d = np.ascontiguousarray(del_ids if del_ids is not None else [], dtype=np.uint32)
        if ins_offsets is None:
            ins_offsets, ins_members = np.zeros(1, np.uint64), np.zeros(0, np.uint32)
        off, mem = _csr_arrays(ins_offsets, ins_members)
        t = C.c_uint64()
        check(lib.hm_serve_submit_update(self._h, graph, ptr(d if len(d) else np.zeros(1, np.uint32), C.c_uint32),
                                         len(d), ptr(off, C.c_uint64),
                                         ptr(mem if len(mem) else np.zeros(1, np.uint32), C.c_uint32), len(off) - 1,
                                         C.byref(t)), "hm_serve_submit_update")
        return t.value

    def submit_count(self, graph: int) -> int:
        t = C.c_uint64()
        check(lib.hm_serve_submit_count(self._h, graph, C.byref(t)), "hm_serve_submit_count")
        return t.value

    def wait(self, ticket: int, cap: int = 1 << 20):
        """(ServeResult, assigned ids) of a request; blocks until served."""
        r = ServeResult()
        ids = np.zeros(max(cap, 1), np.uint32)
        check(lib.hm_serve_wait(self._h, ticket, C.byref(r), ptr(ids, C.c_uint32), cap), "hm_serve_wait")
        return r, ids[: r.n_assigned].copy()

    def drain(self) -> None:
        check(lib.hm_serve_drain(self._h), "hm_serve_drain")

    def stats(self) -> ServeStats:
        s = ServeStats()
        check(lib.hm_serve_stats(self._h, C.byref(s)), "hm_serve_stats")
        return s

    def live_ids(self, graph: int) -> np.ndarray:
        n = C.c_uint32()
        cap = 1 << 22
        out = np.zeros(cap, np.uint32)
        check(lib.hm_serve_live_ids(self._h, graph, ptr(out, C.c_uint32), cap, C.byref(n)), "hm_serve_live_ids")
        return out[: n.value].copy()

    def close(self) -> None:
        if self._h:
            lib.hm_serve_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def classify_static(pattern: int) -> int:
    return lib.hm_classify_static(pattern)


def classify_temporal(pattern: int) -> int:
    return lib.hm_classify_temporal(pattern)
