"""The H2H arena grows in place (virtual memory mapped at its end) and gives
its free tail back under memory pressure. Growth-heavy batch sequences are
checked against the CPU oracle after every batch, with and without a tight
device-memory budget on the context."""
import numpy as np
import pytest

from tests.helpers import csr
from tests.test_dynamic_gpu import Mirror, random_rows

pytestmark = pytest.mark.gpu


def grow_sequence(g, mirror, rng, n_nodes, batches, n_ins, n_del, kmax):
    """Applies the batches; returns how many succeeded before an error (and
    the error, or None). Every successful batch is checked in full."""
    from ipdps26_b200._lib import HmError

    try:
        total = g.count_static30().astype(np.int64)
    except HmError as e:
        return 0, e
    assert total.tolist() == mirror.counts(n_nodes).astype(np.int64).tolist()
    for step in range(batches):
        live = np.array(sorted(mirror.rows), dtype=np.uint32)
        dels = sorted(rng.choice(live, size=min(n_del, len(live)), replace=False).tolist())
        ins_rows = random_rows(rng, n_ins, n_nodes, kmax)
        io, im = csr(ins_rows)
        try:
            ids, delta = g.apply_batch(dels, io, im)
            full = g.count_static30().astype(np.int64)
        except HmError as e:
            return step, e
        want_ids = mirror.apply(dels, ins_rows)
        assert ids.tolist() == want_ids
        want = mirror.counts(n_nodes).astype(np.int64)
        assert full.tolist() == want.tolist(), f"batch {step}"
        assert (total + delta).tolist() == full.tolist(), f"batch {step}: delta"
        total = full
    return batches, None


def test_arena_grows_in_place(ctx):
    from ipdps26_b200 import engine

    rng = np.random.default_rng(11)
    n_nodes = 1000
    rows = random_rows(rng, 6000, n_nodes, 6)
    mirror = Mirror(rows)
    off, mem = csr(rows)
    with engine.Graph(ctx, off, mem, n_nodes) as g:
        a0 = g.info().n_adjacent
        done, err = grow_sequence(g, mirror, rng, n_nodes, batches=6, n_ins=1500, n_del=200, kmax=6)
        assert err is None and done == 6
        assert g.info().n_adjacent > 2 * a0  # the arena had to grow several times


@pytest.mark.parametrize("factor", [1.5, 2.5, 4.0, 16.0])
def test_tight_budget_trims_or_fails_cleanly(factor):
    """Contexts whose budget leaves little room over the built store: the
    arena grows lean, the oriented copy is built after giving back the
    arena's free tail, and a batch that cannot fit fails with HM_ERR_NOMEM
    instead of faulting. Every batch that succeeds is exact, and with room
    enough every batch succeeds."""
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import HM_ERR_NOMEM

    rng = np.random.default_rng(12)
    n_nodes = 800
    rows = random_rows(rng, 5000, n_nodes, 6)
    off, mem = csr(rows)
    with engine.Context(0) as probe:
        with engine.Graph(probe, off, mem, n_nodes) as g:
            g.count_static30()
            used = probe.memory()[0]
    with engine.Context(0, mem_budget_bytes=int(used * factor)) as tight:
        mirror = Mirror(rows)
        try:
            g = engine.Graph(tight, off, mem, n_nodes)
        except Exception as e:  # the store itself may not fit the smallest budgets
            assert getattr(e, "status", None) == HM_ERR_NOMEM, str(e)
            return
        with g:
            done, err = grow_sequence(g, mirror, rng, n_nodes, batches=6, n_ins=1500, n_del=100, kmax=6)
        if err is not None:
            assert err.status == HM_ERR_NOMEM, str(err)
        if factor >= 16.0:
            assert done == 6, str(err)
