"""Host logic of bench.py on the CPU: the config-3 section records where it
stops when the store runs out of memory (a batch or a recount failing with
HM_ERR_NOMEM) and still returns its line, so a memory limit never costs the
whole bench run. The graph is a stand-in that fails on cue; no GPU."""
import argparse

import numpy as np
import pytest


class _Timings:
    update_ms = 12.5
    count_ms = 40.0


class _Info:
    n_adjacent = 1234


class _Ctx:
    def memory(self):
        return (7_000_000_000, 190_000_000_000)


class FakeGraph:
    """Answers like engine.Graph; apply_batch fails at batch fail_batch and
    count_static30 at recount fail_count (1-based), with HM_ERR_NOMEM."""

    def __init__(self, n_live, fail_batch=None, fail_count=None):
        self.live = np.arange(n_live, dtype=np.uint32)
        self.fail_batch, self.fail_count = fail_batch, fail_count
        self.batches = self.counts = 0
        self.ctx = _Ctx()

    def live_ids(self):
        return self.live

    def apply_batch(self, dels, offsets, members):
        from ipdps26_b200._lib import HM_ERR_NOMEM, HmError

        self.batches += 1
        if self.batches == self.fail_batch:
            raise HmError(HM_ERR_NOMEM, "hm_graph_apply_batch", "device budget exceeded")
        n_ins = len(offsets) - 1
        self.live = np.concatenate([np.setdiff1d(self.live, dels), self.live.max() + 1 + np.arange(n_ins)])
        self.live = self.live.astype(np.uint32)
        return None, np.zeros(30, np.int64)

    def count_static30(self):
        from ipdps26_b200._lib import HM_ERR_NOMEM, HmError

        self.counts += 1
        if self.counts == self.fail_count:
            raise HmError(HM_ERR_NOMEM, "hm_count_static30", "device budget exceeded")
        return np.zeros(30, np.uint64)

    def timings(self):
        return _Timings()

    def info(self):
        return _Info()


def _args(batches, every):
    return argparse.Namespace(update_batches=batches, update_edits=40, update_check_every=every)


def _laws():
    from ipdps26_b200 import gen

    return gen.config1(seed=3, n_nodes=300, n_edges=400)


def test_update_section_runs_every_batch_and_check():
    import bench

    g = FakeGraph(400)
    out = bench.update_section(_args(6, 3), g, _laws(), np.zeros(30, np.uint64))
    assert out["batches"] == 6 and out["stopped"] is None
    assert [c["after_batch"] for c in out["recount_checks"]] == [3, 6]
    assert out["delta_sum_equals_full_recount"] is True
    assert len(out["per_batch_ms"]) == 6 and out["per_batch_edits"] == [40] * 6


@pytest.mark.parametrize("fail_batch", [1, 4])
def test_update_section_stops_at_a_failed_batch(fail_batch):
    import bench

    g = FakeGraph(400, fail_batch=fail_batch)
    out = bench.update_section(_args(6, 2), g, _laws(), np.zeros(30, np.uint64))
    assert out["stopped"]["batch"] == fail_batch
    assert "status -3" in out["stopped"]["error"]
    assert out["batches"] == fail_batch - 1
    assert g.batches == fail_batch  # nothing ran after the failure


def test_update_section_stops_at_a_failed_recount():
    import bench

    g = FakeGraph(400, fail_count=2)
    out = bench.update_section(_args(6, 2), g, _laws(), np.zeros(30, np.uint64))
    assert out["stopped"] == {"batch": 4, "in": "recount check", "error": out["stopped"]["error"],
                              "device_gb_in_use": 7.0}
    assert [c["after_batch"] for c in out["recount_checks"]] == [2]
    assert out["batches"] == 4
