"""The oracle's rule for equal timestamps against a line-by-line Python
restatement of THyMe+'s counting loop (THyMe-main/code/main_thymeP.cpp
:188-368) run in a fixed order.

THyMe shuffles its input (read_data.cpp:35-36) before a time sort, so with
ties its counts vary between runs and no fixture can pin them. Without the
shuffle its loop is deterministic: events in (time, input) order, node-sets
numbered as first met in the input. The restatement below follows the loop
as written: window deletion (:228-234), instances (a newest, b, c) with
closed pairs once for b < c and open pairs at a (:243-300), occurrence pairs
with b strictly before c (:313-323), motifs 87-96 (:337-367). One choice is
the restatement's own: THyMe takes an open pair at a in its adjacency-list
order, which depends on its update history; here the node-set met first in
the input plays b, the rule the oracle and the engine use."""
import numpy as np
import pytest

from oracle import oracle
from tests.helpers import csr, random_graph


def _tclass(*args):
    return oracle.lib().hmo_temporal_class(*(int(x) for x in args))


def thyme_loop(rows, times, delta):
    order = sorted(range(len(rows)), key=lambda e: (times[e], e))
    index, sets = {}, []
    static = []
    for r in rows:
        key = frozenset(r)
        if key not in index:
            index[key] = len(sets)
            sets.append(key)
        static.append(index[key])
    occ = [[] for _ in sets]  # E2times: occurrence times inside the window
    count = [0] * 96
    start = 0
    for end in range(len(order)):
        ea = order[end]
        a, ta = static[ea], times[ea]
        while times[order[start]] + delta < ta:  # update_delete
            occ[static[order[start]]].pop(0)
            start += 1
        occ[a].append(ta)  # update_add
        present = [s for s in range(len(sets)) if occ[s]]

        def ov(x, y):
            return len(sets[x] & sets[y])

        nbr_a = [b for b in present if b != a and ov(a, b)]
        inst = []
        for i, b in enumerate(nbr_a):
            seen = set()
            for c in present:
                if c in (a, b) or not ov(b, c):
                    continue
                seen.add(c)
                g = len(sets[a] & sets[b] & sets[c])
                if ov(a, c):
                    if b < c:
                        inst.append((b, c, ov(a, b), ov(b, c), ov(a, c), g))
                else:
                    inst.append((b, c, ov(a, b), ov(b, c), 0, g))
            for c in nbr_a[i + 1:]:
                if c not in seen:
                    p, q = (b, c) if b < c else (c, b)
                    inst.append((p, q, ov(a, p), 0, ov(a, q), 0))
        sa = len(sets[a])
        for b, c, cab, cbc, cac, g in inst:
            sb, sc = len(sets[b]), len(sets[c])
            bc = sum(1 for x in occ[b] for y in occ[c] if x < y)
            count[_tclass(sb, sc, sa, cbc, cac, cab, g)] += bc
            count[_tclass(sc, sb, sa, cbc, cab, cac, g)] += len(occ[b]) * len(occ[c]) - bc
        earlier = occ[a][:-1]
        for b in nbr_a:
            cab, sb = ov(a, b), len(sets[b])
            ab = sum(1 for x in earlier for y in occ[b] if x < y)
            count[_tclass(sa, sb, sa, cab, cab, sa, cab)] += ab
            count[_tclass(sb, sa, sa, cab, sa, cab, cab)] += len(earlier) * len(occ[b]) - ab
            count[_tclass(sb, sb, sa, sb, cab, cab, cab)] += len(occ[b]) * (len(occ[b]) - 1) // 2
        if len(earlier) >= 2:
            count[95] += len(earlier) * (len(earlier) - 1) // 2
    return count


@pytest.mark.parametrize("seed", range(6))
def test_oracle_tie_rule_is_thymes_loop_in_input_order(seed):
    rng = np.random.default_rng(40 + seed)
    for _ in range(40):
        n_nodes = int(rng.integers(3, 8))
        off, mem = random_graph(rng, int(rng.integers(3, 11)), n_nodes, 3)
        rows = [sorted(set(mem[off[i]:off[i + 1]].tolist())) for i in range(len(off) - 1)]
        if rng.random() < 0.5:
            for i in range(0, len(rows), 3):
                rows[i] = rows[max(0, i - 1)]
        times = rng.integers(0, 4, size=len(rows)).astype(np.int64)
        off, mem = csr(rows)
        for delta in (0, 1, 3, 10):
            want = thyme_loop(rows, times.tolist(), delta)
            assert oracle.temporal96(off, mem, times, delta).tolist() == want, (rows, times.tolist(), delta)
