"""One picture in row strips across ranks (unround.strips), without a GPU: the partition gives
every band to one rank and each rank at least the halo's bands; the swap schedule sends each
halo row from the rank that owns it; and with two and three gloo ranks on the CPU, each rank's
planes -- rows marked by their row of the whole canvas -- come out of the swap with every halo
row the owner's."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def test_partition_and_schedule():
    from unround.strips import HALO_BANDS, exchanges, partition

    for bands, ranks in [(4, 2), (9, 2), (10, 3), (40, 8), (7, 3)]:
        parts = partition(bands, ranks)
        owned = [b for p in parts for b in range(p.first, p.end)]
        assert owned == list(range(bands))
        for p in parts:
            assert p.end - p.first >= HALO_BANDS
            assert p.low == max(0, p.first - HALO_BANDS) and p.high == min(bands, p.end + HALO_BANDS)
        rows = 16
        for sender, s_row, receiver, r_row, count in exchanges(parts, rows):
            s, r = parts[sender], parts[receiver]
            assert abs(sender - receiver) == 1 and count > 0 and count % rows == 0
            # The rows sent are the sender's own, and land where the receiver keeps the same rows.
            first_band = s.low + s_row // rows
            assert s.first <= first_band and first_band + count // rows <= s.end
            assert r.low + r_row // rows == first_band
            assert not (r.first <= first_band < r.end)
    with pytest.raises(ValueError):
        partition(3, 2)


def _rank(rank: int, world: int, port: int, bands: int, results) -> None:
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from unround.strips import exchange, partition

        rows, columns = 8, 5
        parts = partition(bands, world)
        mine = parts[rank]
        height = (mine.high - mine.low) * rows
        # Each plane's value: its plane number, its row of the whole canvas, and who holds it
        # (-1 in the halo before the swap).
        planes = []
        for k in range(3):
            plane = torch.full((height, columns), -1.0)
            for local in range(height):
                band = mine.low + local // rows
                if mine.first <= band < mine.end:
                    plane[local] = 1000.0 * k + (mine.low * rows + local)
            planes.append(plane)
        exchange(planes, parts, rank, rows)
        results[rank] = [p.numpy().copy() for p in planes]
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world, bands", [(2, 6), (3, 9)])
def test_gloo_ranks_swap_their_halos(world, bands):
    from unround.strips import partition

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank, args=(world, port, bands, results), nprocs=world, join=True, start_method="spawn")
    rows = 8
    for rank, part in enumerate(partition(bands, world)):
        for k, plane in enumerate(results[rank]):
            expected = 1000.0 * k + part.low * rows + np.arange(plane.shape[0])
            np.testing.assert_array_equal(plane, np.repeat(expected[:, None], plane.shape[1], axis=1))
