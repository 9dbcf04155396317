"""One picture in row strips (unround.strips.solve_in_strips): the strips' solvers on one GPU with
their halo rows swapped after every iteration, against the whole picture solved at once
(unround_solve): the canvas to binary32 rounding (rel L2 <= 1e-5, max |difference| <= 1e-3 on
0-255), grey and colour, TV and TGV, heights that are not whole bands, two to four strips; and
the records the strips add up across the ranks (every 10 iterations, TGV's scaling and partial
gap among them) within 1e-9 of the whole solve's, with the same stop at a tolerance."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    ("grey-tgv-2", "grey", (150, 96), ["--method", "tgv"], 2),
    ("grey-tv-3", "grey", (203, 77), ["--method", "tv", "--alpha", "1.5"], 3),
    ("colour420-tgv-2", "colour", (161, 120), ["--method", "tgv"], 2),
    ("colour420-tv-apart-4", "colour", (290, 88), ["--method", "tv", "--channels", "apart"], 4),
]


@pytest.mark.parametrize("name, kind, shape, options, strips", CASES, ids=[c[0] for c in CASES])
def test_strips_equal_the_whole_solve(name, kind, shape, options, strips):
    from unround import native, synthetic
    from unround.strips import solve_in_strips

    make = synthetic.grey if kind == "grey" else synthetic.colour
    image = make(*shape, quality=60, seed=len(name), noise=2.0).image
    given = [*options, "--iterations", "60", "--tolerance", "0", "--record-every", "0"]
    whole = native.solve(image, given).canvas
    parts = solve_in_strips(image, given, strips).canvas
    assert parts.shape == whole.shape
    difference = parts - whole
    assert np.linalg.norm(difference) / np.linalg.norm(whole) <= 1e-5, name
    assert np.abs(difference).max() <= 1e-3, name


def test_the_distributed_form_on_one_rank():
    # solve_strip under torch.distributed with NCCL at one rank (this pool gives one GPU a call):
    # the driver, the state's planes aliased as device tensors and the swap's (empty) schedule.
    import os
    import socket

    import torch.distributed as dist

    from unround import native, synthetic
    from unround.strips import solve_strip

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    image = synthetic.grey(120, 64, quality=50, seed=9, noise=2.0).image
    given = ["--method", "tgv", "--iterations", "30", "--tolerance", "0", "--record-every", "0"]
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        mine = solve_strip(image, given).canvas
    finally:
        dist.destroy_process_group()
    whole = native.solve(image, given).canvas
    np.testing.assert_allclose(mine, whole, rtol=0, atol=1e-3)
    assert np.linalg.norm(mine - whole) / np.linalg.norm(whole) <= 1e-5


RECORDED = [
    ("grey-tgv-partial-2", "grey", (150, 96), ["--method", "tgv", "--partial-radius", "4"], 2),
    ("colour420-tgv-3", "colour", (240, 88), ["--method", "tgv"], 3),
    ("grey-tv-2", "grey", (130, 72), ["--method", "tv"], 2),
]


@pytest.mark.parametrize("name, kind, shape, options, strips", RECORDED, ids=[c[0] for c in RECORDED])
def test_strips_records_equal_the_whole_solve(name, kind, shape, options, strips):
    from unround import native, synthetic
    from unround.strips import solve_in_strips

    make = synthetic.grey if kind == "grey" else synthetic.colour
    image = make(*shape, quality=50, seed=len(name), noise=2.0).image
    given = [*options, "--iterations", "60", "--tolerance", "0", "--record-every", "10"]
    whole = native.solve(image, given)
    parts = solve_in_strips(image, given, strips)
    mine, theirs = parts.history, whole.result.history
    np.testing.assert_array_equal(mine.iterations, theirs.iterations)
    for column in ("primal", "dual", "scaling", "partial_gap"):
        np.testing.assert_allclose(getattr(mine, column), getattr(theirs, column), rtol=1e-9, atol=0,
                                   err_msg=f"{name}: {column}")
    assert parts.iterations == whole.result.iterations and parts.stop == int(whole.result.stop)
    assert np.linalg.norm(parts.canvas - whole.canvas) / np.linalg.norm(whole.canvas) <= 1e-5


def test_strips_stop_at_a_tolerance_with_the_whole_solve():
    from unround import native, synthetic
    from unround.strips import solve_in_strips

    image = synthetic.grey(160, 120, quality=40, seed=71, noise=2.0).image
    probe = ["--method", "tgv", "--iterations", "200", "--tolerance", "0", "--record-every", "10"]
    history = native.solve(image, probe).result.history
    per_sample = history.gap / (image.height * image.width)  # one channel, whole MCUs
    # A tolerance between the records of iterations 50 and 60: the solve stops at 60.
    assert per_sample[6] < per_sample[5] and np.all(per_sample[:6] > per_sample[6])
    tolerance = float(np.sqrt(per_sample[6] * per_sample[5]))
    given = ["--method", "tgv", "--iterations", "200", "--tolerance", repr(tolerance), "--record-every", "10"]
    whole = native.solve(image, given)
    parts = solve_in_strips(image, given, 2)
    assert whole.result.stop is native.Stop.CONVERGED and whole.result.iterations == 60
    assert parts.stop == 1 and parts.iterations == 60
    np.testing.assert_allclose(parts.history.primal, whole.result.history.primal, rtol=1e-9, atol=0)
    assert np.linalg.norm(parts.canvas - whole.canvas) / np.linalg.norm(whole.canvas) <= 1e-5


def test_nccl_exchange_equals_the_local_one():
    """The library's swap through NCCL (unround_b200_strip_run, torch's communicator at one rank,
    a strip exchanging rows with itself) against its swap of device copies
    (unround_b200_strip_exchange_local): after each of five iterations, every state plane bit for
    bit, and the exchanged rows equal to their sources."""
    import os
    import socket

    import torch
    import torch.distributed as dist

    from unround import synthetic
    from unround.strips import StripSolver, _communicator, exchange_local

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    image = synthetic.colour(161, 120, quality=60, seed=5, noise=2.0).image
    given = ["--method", "tgv", "--iterations", "20", "--tolerance", "0", "--record-every", "0"]
    # (sender, its first row, receiver, its first row, rows): disjoint sources and targets.
    swaps = [(0, 0, 0, 48, 16), (0, 96, 0, 16, 8)]
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        comm = _communicator(None)
        assert comm is not None, "torch exposes no NCCL communicator"
        through_nccl, local = StripSolver(image, given), StripSolver(image, given)
        through_nccl.run(5, 0, swaps, comm)
        for _ in range(5):
            local.run(1)
            exchange_local([local], swaps)
        torch.cuda.synchronize()
        mine = [t.clone() for t in through_nccl.planes()]
        theirs = [t.clone() for t in local.planes()]
    finally:
        dist.destroy_process_group()
    assert len(mine) == len(theirs) == 8 * 3
    for k, (a, b) in enumerate(zip(mine, theirs)):
        assert torch.equal(a, b), f"plane {k}"
        assert torch.equal(a[48:64], a[0:16]) and torch.equal(a[16:24], a[96:104]), f"plane {k}"


def test_exchanges_refused():
    """The library's swaps refuse what they cannot do, before touching the device: rows beyond a
    strip's canvas, a strip index beyond those given, an exchange of this rank with no NCCL
    communicator, and the strip's last iteration (its record's or _finish's)."""
    from unround import native, synthetic
    from unround.strips import StripSolver, exchange_local

    image = synthetic.grey(96, 64, quality=50, seed=3, noise=2.0).image
    given = ["--method", "tgv", "--iterations", "10", "--tolerance", "0", "--record-every", "0"]
    solver = StripSolver(image, given)
    with pytest.raises(native.UnroundError, match="does not hold its rows") as caught:
        solver.run(0, 0, [(0, 0, 0, 90, 16)], None)
    assert caught.value.status is native.Status.ARGUMENT
    with pytest.raises(native.UnroundError, match="beyond the 1 given"):
        exchange_local([solver], [(0, 0, 1, 16, 8)])
    with pytest.raises(native.UnroundError, match="NCCL communicator"):
        solver.run(1, 0, [(0, 0, 1, 16, 8)], None)
    with pytest.raises(native.UnroundError, match="last iteration"):
        solver.run(10)
    solver.run(9)  # the rest is allowed: iterations 1 .. 9, no exchanges


def test_the_distributed_form_records_on_one_rank():
    """solve_strip at one NCCL rank with records every 10 iterations: the iterations between
    records as one library call each (StripSolver.run on torch's communicator), the records
    gathered, and the history and stop of the whole solve."""
    import os
    import socket

    import torch.distributed as dist

    from unround import native, synthetic
    from unround.strips import solve_strip

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    image = synthetic.colour(144, 96, quality=50, seed=11, noise=2.0).image
    given = ["--method", "tgv", "--iterations", "45", "--tolerance", "0", "--record-every", "10"]
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        mine = solve_strip(image, given)
    finally:
        dist.destroy_process_group()
    whole = native.solve(image, given)
    theirs = whole.result.history
    np.testing.assert_array_equal(mine.history.iterations, theirs.iterations)
    for column in ("primal", "dual", "scaling"):
        np.testing.assert_allclose(getattr(mine.history, column), getattr(theirs, column), rtol=1e-9, atol=0,
                                   err_msg=column)
    assert mine.iterations == 45 and mine.stop == int(whole.result.stop)
    assert np.linalg.norm(mine.canvas - whole.canvas) / np.linalg.norm(whole.canvas) <= 1e-5
