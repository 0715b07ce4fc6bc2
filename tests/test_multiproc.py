"""The multi-rank path on the CPU: world size 2 over gloo.

Each rank counts its share of the owner hyperedges (the oracle's shard, the
same owner rule the GPU shards use), the partials meet in
``shard.allreduce_counts``, and every rank must end with the full count.
The GPU side of the split (``count_static30_shard`` partials summing to the
full count) is covered in test_static_gpu.py.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.helpers import random_graph, static_case

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, cases, out_dir):
    import datetime

    import torch.distributed as dist

    from ipdps26_b200 import shard
    from oracle import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {}
        for name, (off, mem, n_nodes) in cases.items():
            part = oracle.static30_shard(off, mem, n_nodes, rank, world)
            res[name] = (part, shard.allreduce_counts(part, dist))
        # exact modulo 2^64 for values above the int64 range
        big = np.array([2**63 + 5, 2**64 - 1 - rank, 7], np.uint64)
        res["big"] = (big, shard.allreduce_counts(big, dist))
        res["max"] = shard.max_over_ranks(1.5 + rank, dist)
        # each rank tuned its own schedule; rank 0's is the one all use
        mine = (64, 2048, 0, 1024) if rank == 0 else (128, 2048, 128, 2048)
        res["schedule"] = shard.agree_schedule(mine, dist)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array([res], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _cases():
    rng = np.random.default_rng(7)
    cases = {}
    off, mem = random_graph(rng, 150, 40, 8)
    cases["random"] = (off, mem, 40)
    h = static_case(dict(seed=11, n_nodes=1000, n_edges=2000, k_min=2, k_max=25, size_exp=2.5, pop_exp=1.2,
                         pop_offset=0.0))
    cases["c1law-2k"] = (h.offsets, h.members, h.n_nodes)
    return cases


def test_sharded_count_all_reduce_over_gloo(tmp_path):
    from oracle import oracle

    cases = _cases()
    mp.start_processes(_rank_main, args=(WORLD, _free_port(), cases, str(tmp_path)), nprocs=WORLD, join=True,
                       start_method="spawn")
    results = [np.load(tmp_path / f"rank{r}.npy", allow_pickle=True)[0] for r in range(WORLD)]
    for name, (off, mem, n_nodes) in cases.items():
        full = oracle.static30(off, mem, n_nodes)
        parts = [results[r][name][0] for r in range(WORLD)]
        # the owner split is a partition: no triple counted twice or lost
        assert np.array_equal(parts[0] + parts[1], full), name
        assert all(p.sum() > 0 for p in parts), name
        for r in range(WORLD):
            assert np.array_equal(results[r][name][1], full), (name, r)
    want_big = (np.array([2**63 + 5, 2**64 - 1, 7], np.uint64) * np.uint64(2)) - np.array([0, 1, 0], np.uint64)
    for r in range(WORLD):
        assert np.array_equal(results[r]["big"][1], want_big)
        assert results[r]["max"] == pytest.approx(1.5 + WORLD - 1)
        assert results[r]["schedule"] == (64, 2048, 0, 1024)


def test_owner_shards_cover_every_owner_once():
    from ipdps26_b200 import shard

    ids = np.arange(1000, dtype=np.uint64)
    for world in (1, 2, 3, 8):
        s = shard.owner_shard(ids, world)
        assert s.min() == 0 and s.max() == world - 1
        assert np.bincount(s, minlength=world).sum() == len(ids)
