"""The allocation-free touched-triple count, for callers that cannot call
cudaMalloc while they run (a serving loop that must not block on the
allocator, code held to a fixed memory reservation). It must give the same
30 counts as the allocating hm_count_touching30, call after call, from
device buffers owned by the caller. This file is collected last so that a
failure here does not hide the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(g, ids_dev, n, out_dev):
    from ipdps26_b200 import engine
    from ipdps26_b200._lib import check, lib

    fn = lib.hm_count_touching30_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    check(fn(g.handle, C.c_void_p(ids_dev), n, C.c_void_p(out_dev), None), "hm_count_touching30_noalloc")
    assert engine  # the engine module binds the rest of the ABI


def test_noalloc_matches_allocating_call_twice_in_a_row():
    import torch

    from ipdps26_b200 import engine, gen

    h = gen.static(gen.config1(seed=21, n_nodes=700, n_edges=1500))
    with engine.Context(0) as ctx, engine.Graph.from_hypergraph(ctx, h) as g:
        rng = np.random.default_rng(21)
        out = torch.zeros(30, dtype=torch.int64, device="cuda:0")
        for n in (40, 400):  # two calls in a row, on different id sets
            ids = np.unique(rng.choice(h.n_edges, size=n, replace=False)).astype(np.uint32)
            want = g.count_touching30(ids)
            ids_dev = torch.from_numpy(ids.view(np.int32)).to("cuda:0")
            out.fill_(-1)
            torch.cuda.synchronize()
            _noalloc(g, ids_dev.data_ptr(), len(ids), out.data_ptr())
            got = out.cpu().numpy().view(np.uint64)
            assert got.tolist() == want.tolist(), n
