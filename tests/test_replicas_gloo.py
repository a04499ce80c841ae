"""The multi-GPU path is replicas: each rank reconstructs its own slices, and
timings are reduced max-over-ranks.  Exercised here with two gloo ranks on the
CPU (the oracle stands in for the device backprojection)."""
import os
import socket

import numpy as np
import pytest

from ctas_b200.replicas import shard


def test_shard_covers_every_item_once():
    for n in (0, 1, 7, 256, 1000):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shard(n, r, world)]
            assert got == list(range(n))
            sizes = [len(shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    import oracle as O
    from ctas_b200.replicas import max_over_ranks, shard as shard_
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        S, N, W = 5, 30, 32
        rng = np.random.default_rng(0)
        stack = rng.standard_normal((S, N, W)).astype(np.float32)
        tab = O.angle_table(180.0, N)
        mine = shard_(S, rank, world)
        parts = {s: O.bp_compat(stack[s], tab, 1.0, 1.0) for s in mine}
        t = max_over_ranks(float(rank + 1))
        gathered = [None] * world
        dist.all_gather_object(gathered, parts)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            assert sorted(merged) == list(range(S))
            for s in range(S):
                assert np.array_equal(merged[s], O.bp_compat(stack[s], tab, 1.0, 1.0))
            assert t == float(world)
            with open(os.path.join(out_dir, "ok"), "w") as f:
                f.write("ok")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reconstruct_their_shards(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    assert (tmp_path / "ok").exists()
