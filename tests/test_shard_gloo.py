"""Multi-rank logic of bench.py on CPU: two gloo ranks split a batch of planes
into disjoint slices covering it, get distinct seeds, and agree on the max
time -- the same calls the NCCL run makes, without a GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_items, out):
    import torch
    import torch.distributed as dist
    from isp_mw_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard.shard(list(range(n_items)), rank, world)
    seeds = [shard.plane_seed(rank, s, k) for s in range(4) for k in range(4)]
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, seeds))
    t = shard.max_over_ranks(10.0 + rank)
    dist.barrier()
    out[rank] = (gathered, t)
    dist.destroy_process_group()


@pytest.mark.parametrize("n_items", [0, 1, 7, 64])
def test_two_gloo_ranks_shard_and_reduce(n_items):
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), n_items, out), nprocs=world,
                       join=True, start_method="spawn")
    for rank in range(world):
        gathered, t = out[rank]
        assert t == 10.0 + world - 1  # max over ranks
        items = [i for g in gathered for i in g[0]]
        assert sorted(items) == list(range(n_items))  # disjoint and complete
        seeds = [s for g in gathered for s in g[1]]
        assert len(seeds) == len(set(seeds))


def test_shard_range_balance():
    from isp_mw_b200 import shard
    for n in range(0, 40):
        for w in range(1, 9):
            sizes = [shard.shard_range(n, r, w)[1] - shard.shard_range(n, r, w)[0] for r in range(w)]
            assert sum(sizes) == n and max(sizes) - min(sizes) <= 1
