"""Full-size parity: the configurations exactly as specified, against the
reference's own counters run on them (tests/golden/full_golden.json, written
by `make_golden.py --full`: MoCHy main_exact_par, THyMe+ main_thymeP)."""
import json

import pytest

from tests.helpers import GOLDEN, digest, static_case, temporal_case

pytestmark = pytest.mark.gpu

FULL = json.loads((GOLDEN / "full_golden.json").read_text()) if (GOLDEN / "full_golden.json").exists() else {}


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_size_matches_reference(ctx, name):
    from ipdps26_b200 import engine

    rec = FULL[name]
    if rec["kind"] == "static":
        h = static_case(rec["params"])
        assert digest(h) == rec["sha256"]
        with engine.Graph.from_hypergraph(ctx, h) as g:
            assert g.count_static().tolist() == rec["counts26"]
    else:
        h = temporal_case(rec["params"])
        assert digest(h) == rec["sha256"]
        with engine.Graph.from_hypergraph(ctx, h) as g:
            for d, want in rec["counts96"].items():
                assert g.count_temporal(int(d)).tolist() == want, d
