"""Multi-rank host logic of bench.py on CPU: world size 2 over gloo (the GPU run uses one rank per
GPU over NCCL with the same calls)."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        got = bench.reduce_max((1.0 + rank, 10.0 - rank, 3.5), world, torch.device("cpu"))
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    port = 29500 + (os.getpid() % 2000)
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 10.0, 3.5)


def test_rank_shards_are_disjoint():
    sys.path.insert(0, str(ROOT))
    import bench
    B = 10000
    spans = []
    for r in range(8):
        ri, seed = bench.rank_shard(r, B)
        # key i of a rank uses counter ri + 2i + 1 (odd), messages use their own seeds
        spans.append((ri + 1, ri + 2 * (B - 1) + 1, seed))
    for a in range(8):
        for b in range(a + 1, 8):
            assert spans[a][1] < spans[b][0] or spans[b][1] < spans[a][0]
            assert spans[a][2] != spans[b][2]


def test_reduce_max_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_max((1.5, 2.5), 1, None) == (1.5, 2.5)
