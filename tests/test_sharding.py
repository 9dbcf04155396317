"""Pictures across ranks (unround.sharding), without a GPU: the shares partition the pictures and
balance their pixels; with two gloo ranks on the CPU, the slowest rank's time and the sum over
ranks are every rank's, and each rank's share of a mix is what the split says."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def test_shares_partition_and_balance():
    from unround.sharding import shard

    weights = [256 * 256, 2048 * 2048, 512 * 768, 1024 * 1024, 256 * 2048, 1536 * 1536, 640 * 480]
    for world in (1, 2, 3, 4, 8):
        shares = shard(weights, world)
        assert sorted(n for s in shares for n in s) == list(range(len(weights)))
        loads = [sum(weights[n] for n in s) for s in shares]
        # Greedy largest-first: the slowest rank has at most the ideal share plus the largest picture.
        assert max(loads) <= sum(weights) / world + max(weights)
    with pytest.raises(ValueError):
        shard(weights, 0)


def _rank(rank: int, world: int, port: int, results) -> None:
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from unround import synthetic
        from unround.sharding import max_over_ranks, rank_and_world, shard, sum_over_ranks

        me, size = rank_and_world()
        mix = synthetic.mix(6, seed=4, smallest=32, largest=96, iterations=3)
        shares = shard([e.image.height * e.image.width for e in mix], size)
        mine = shares[me]
        pixels = sum(mix[n].image.height * mix[n].image.width for n in mine)
        results[me] = (max_over_ranks(10.0 * (me + 1)), sum_over_ranks(pixels), mine, pixels)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank, args=(2, port, results), nprocs=2, join=True, start_method="spawn")
    assert set(results.keys()) == {0, 1}
    total = results[0][3] + results[1][3]
    for rank in (0, 1):
        slowest, pixels, mine, _ = results[rank]
        assert slowest == 20.0
        assert pixels == total
    assert sorted(results[0][2] + results[1][2]) == list(range(6))
