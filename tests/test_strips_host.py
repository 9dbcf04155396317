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


class _FakeSolver:
    """A strip's solver without a GPU: its record sums a function of the rank and the iteration
    (the dual value nearing the primal as the iterations go), its planes CPU tensors."""

    def __init__(self, rank: int, height: int) -> None:
        import torch

        self.rank, self.done, self.rows = rank, 0, None
        self._planes = [torch.zeros((height, 4)) for _ in range(3)]

    @staticmethod
    def plan():
        from unround.strips import StripPlan

        return StripPlan(iterations=40, record_every=5, tolerance=0.005, relative_tolerance=0.0,
                         partial_tolerance=0.0, partial_radius=3.0, alpha=1.0, alpha1=1.0, alpha0=2.0, tgv=True)

    def set_rows(self, first: int, end: int) -> None:
        self.rows = (first, end)

    def step(self, iterations: int = 1) -> None:
        self.done += iterations

    def planes(self) -> list:
        return self._planes

    @staticmethod
    def firsts(rank: int, done: int) -> list[float]:
        # G, first-order norms, second-order norms, largest |div2 r~|, samples.
        return [100.0 + rank, 50.0 * (rank + 1), 20.0 + rank, 1.5 + 0.5 * rank + done * 0.01, 64.0 * (rank + 1)]

    @staticmethod
    def seconds(rank: int, done: int, theta: float) -> list[float]:
        # The dual's conjugates (the dual value nears the primal, 433, as the iterations go), the
        # partial gap's conjugates, its residual.
        return [-(216.5 - 10.0 / (1 + done)), -(200.0 + rank), 0.25 * (rank + 1) * theta]

    def record(self, advance: bool) -> list[float]:
        if advance:
            self.done += 1
        return self.firsts(self.rank, self.done)

    def record_duals(self, theta: float) -> list[float]:
        return self.seconds(self.rank, self.done, theta)

    def result(self, stop: int) -> tuple[int, int]:
        return self.done, stop


def _records_rank(rank: int, world: int, port: int, bands: int, results) -> None:
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from unround.strips import drive_rank, partition

        rows = 8
        parts = partition(bands, world)
        solver = _FakeSolver(rank, (parts[rank].high - parts[rank].low) * rows)
        result, records, iterations, stop = drive_rank(solver, parts, rank, rows)
        results[rank] = (result, records, iterations, stop, solver.rows)
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_take_the_same_records_and_stop():
    """Two gloo ranks gather their record sums: both take the records that the sums of every
    rank make (combine, in rank order), count only their own rows, and stop together at the first
    record whose gap per sample meets the tolerance."""
    from unround.strips import _met, combine, partition

    world, bands = 2, 6
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_records_rank, args=(world, port, bands, results), nprocs=world, join=True,
                       start_method="spawn")
    plan = _FakeSolver.plan()
    expected, stop_at = [], None
    for n in [0, *range(5, plan.iterations + 1, 5)]:
        firsts = [_FakeSolver.firsts(r, n) for r in range(world)]
        values, samples = combine(plan, firsts, lambda theta: [_FakeSolver.seconds(r, n, theta) for r in range(world)])
        expected.append((n, 0.0, *values))
        if _met(plan, values, samples):
            stop_at = n
            break
    assert stop_at is not None and 0 < stop_at < plan.iterations
    parts = partition(bands, world)
    for rank in range(world):
        (done, stop), records, iterations, stop_reason, rows = results[rank]
        assert records == expected
        assert iterations == stop_at and done == stop_at and stop == 1 and stop_reason == 1
        assert rows == ((parts[rank].first - parts[rank].low) * 8, (parts[rank].end - parts[rank].low) * 8)
    # TGV's scaling is alpha1 over the largest |div2 r~| of every rank's, not of one.
    largest = max(_FakeSolver.firsts(r, 5)[3] for r in range(world))
    assert expected[1][4] == (plan.alpha1 / largest if largest > plan.alpha1 else 1.0)


def test_drive_makes_the_iterations_between_records_in_one_run():
    """The loop's calls: the start's swap, a record at 0, then each stretch of iterations between
    two records as one run(k) (each iteration followed by its swap inside), the recorded iteration
    (made by the record) and its swap; the last iteration is always recorded."""
    from unround.strips import StripPlan, _drive

    plan = StripPlan(iterations=25, record_every=10, tolerance=0.0, relative_tolerance=0.0, partial_tolerance=0.0,
                     partial_radius=None, alpha=1.0, alpha1=1.0, alpha0=2.0, tgv=False)
    calls = []

    def firsts_of(advance):
        calls.append(("record", advance))
        return [[1.0, 2.0, 0.0, 0.0, 4.0]]

    records, iterations, stop = _drive(plan, lambda k: calls.append(("run", k)), firsts_of,
                                       lambda theta: [[-1.0, 0.0, 0.0]])
    assert calls == [("run", 0), ("record", False), ("run", 9), ("record", True), ("run", 0), ("run", 9),
                     ("record", True), ("run", 0), ("run", 4), ("record", True), ("run", 0)]
    assert [r[0] for r in records] == [0, 10, 20, 25] and iterations == 25 and stop == 2
    # Without records between: one stretch, then the last iteration's record.
    plan = StripPlan(iterations=7, record_every=0, tolerance=0.0, relative_tolerance=0.0, partial_tolerance=0.0,
                     partial_radius=None, alpha=1.0, alpha1=1.0, alpha0=2.0, tgv=False)
    calls.clear()
    records, iterations, stop = _drive(plan, lambda k: calls.append(("run", k)), firsts_of,
                                       lambda theta: [[-1.0, 0.0, 0.0]])
    assert calls == [("run", 0), ("run", 6), ("record", True), ("run", 0)]
    assert [r[0] for r in records] == [7] and iterations == 7 and stop == 2
