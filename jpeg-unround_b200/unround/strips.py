"""One picture solved in row strips across ranks (no counterpart in the reference, which splits a
picture into strips across threads: docs/math.md of JPEG-Unround, the strip decomposition).

The picture's MCU bands (8 x max v canvas rows each) are split among the ranks; each rank solves
its own canvas -- its bands and HALO_BANDS bands either side (fewer at the picture's ends) --
with the ordinary kernels, and after the start and after every iteration the halo rows of the
state (x, p and for TGV w and r, every channel) are overwritten with the neighbours' own rows.
Within one iteration a difference from the whole picture's solve can start only at a strip's
edge (where the kernels see an end of the canvas, or a block whose neighbours are missing) and
spreads at most a row and a band inward, so with two halo bands the rows a rank owns are the
whole solve's, iteration after iteration; the last iteration and the result are each strip's,
and the owned rows of the canvases make the picture's canvas.

  partition        which bands each rank owns and which its canvas holds
  sub_image        a strip's bands of a JPEG file's components, as an Image
  exchanges        the rows each neighbour pair swaps: (sender, sender's first row, receiver,
                   receiver's first row, rows)
  exchange         the swap over torch.distributed from Python (gloo on the CPU; NCCL where the
                   library's own swap cannot be used)
  combine          a record of the picture from every rank's sums
  solve_in_strips  the whole solve with the strips in one process on one GPU (the ranks
                   emulated, the swaps device copies between them inside the library), for tests
                   and one device
  solve_strip      a rank's part of it under torch.distributed (one process per GPU; the
                   iterations between records and their swaps one library call, NCCL sends and
                   receives on the strip's stream with no host wait)
"""

from __future__ import annotations

import ctypes
import math
from collections.abc import Callable, Sequence
from dataclasses import dataclass
from typing import Final

import numpy as np
import numpy.typing as npt

from unround import jpegio

HALO_BANDS: Final = 2


@dataclass(frozen=True)
class Strip:
    """A rank's strip: the bands it owns, [first, end), and those its canvas holds, [low, high)."""

    rank: int
    first: int
    end: int
    low: int
    high: int


def band_rows(image: jpegio.Image) -> int:
    """Canvas rows of an MCU band."""
    return 8 * image.max_v_samp_factor


def band_count(image: jpegio.Image) -> int:
    rows = band_rows(image)
    return -(-image.height // rows)


def partition(bands: int, ranks: int, halo: int = HALO_BANDS) -> list[Strip]:
    """The bands split as evenly as whole bands allow; every rank owns at least `halo` bands, so
    that each halo lies in one neighbour's own bands."""
    if ranks < 1:
        raise ValueError("at least one rank")
    if bands < ranks * halo:
        raise ValueError(f"{bands} bands cannot give {ranks} ranks {halo} bands each")
    strips = []
    for rank in range(ranks):
        first, end = rank * bands // ranks, (rank + 1) * bands // ranks
        strips.append(Strip(rank, first, end, max(0, first - halo), min(bands, end + halo)))
    return strips


def sub_image(image: jpegio.Image, strip: Strip) -> jpegio.Image:
    """The strip's canvas as a picture of its own: the components' block rows of its bands, and
    the picture's rows within them."""
    rows = band_rows(image)
    components = []
    for c in image.components:
        v = c.v_samp_factor
        blocks = np.ascontiguousarray(c.coefficients[strip.low * v : min(strip.high * v, c.height_in_blocks)])
        components.append((blocks, c.quant_table.reshape(64), c.h_samp_factor, v))
    height = min(image.height, strip.high * rows) - strip.low * rows
    return jpegio.image_of(height, image.width, image.color_space, components)


def exchanges(strips: list[Strip], rows: int, halo: int = HALO_BANDS) -> list[tuple[int, int, int, int, int]]:
    """Each swap of halo rows: (sender, its first local row, receiver, its first local row, rows)."""
    out = []
    for upper, lower in zip(strips, strips[1:]):
        # The upper strip's last own bands to the lower's halo above; the lower's first own bands
        # to the upper's halo below.
        lo = max(upper.first, upper.end - halo)
        out.append((upper.rank, (lo - upper.low) * rows, lower.rank, (lo - lower.low) * rows, (upper.end - lo) * rows))
        hi = min(lower.end, lower.first + halo)
        out.append((lower.rank, (lower.first - lower.low) * rows, upper.rank, (lower.first - upper.low) * rows,
                    (hi - lower.first) * rows))
    return out


def exchange(planes: list, strips: list[Strip], rank: int, rows: int, group: object = None,
             halo: int = HALO_BANDS) -> None:
    """This rank's part of the swaps: its planes (2D tensors, rows x columns, on the CPU for gloo
    or the device for NCCL) sent as one packed tensor to each neighbour and their rows received
    into its halos. Every rank posts its sends and receives together, so no order can deadlock."""
    import torch
    import torch.distributed as dist

    requests, received = [], []
    for sender, s_row, receiver, r_row, count in exchanges(strips, rows, halo):
        if sender == rank:
            packed = torch.stack([p[s_row : s_row + count] for p in planes]).contiguous()
            requests.append(dist.isend(packed, receiver, group=group))
        elif receiver == rank:
            buffer = torch.empty((len(planes), count, planes[0].shape[1]), dtype=planes[0].dtype,
                                 device=planes[0].device)
            requests.append(dist.irecv(buffer, sender, group=group))
            received.append((buffer, r_row, count))
    for request in requests:
        request.wait()
    for buffer, r_row, count in received:
        for p, part in zip(planes, buffer):
            p[r_row : r_row + count].copy_(part)


# --- The strips' solvers through the C interface. -------------------------------------------


class _DevicePlane:
    """A device plane as __cuda_array_interface__ describes it (for torch.as_tensor, no copy)."""

    def __init__(self, pointer: int, rows: int, columns: int, pitch: int) -> None:
        self.__cuda_array_interface__ = {"shape": (rows, columns), "typestr": "<f4", "data": (pointer, False),
                                         "strides": (4 * pitch, 4), "version": 3}


class StripSolver:
    """A strip's solver (unround_b200_strip_*): started on creation."""

    def __init__(self, image: jpegio.Image, options: list[str]) -> None:
        from unround import native

        self._native = native
        self._library = native._library()
        _bind(self._library)
        self._settings = native._Settings(options)
        given, self._kept = native._input_of(image)
        handle = ctypes.c_void_p()
        message = ctypes.create_string_buffer(native._MESSAGE)
        status = self._library.unround_b200_strip_new(ctypes.byref(given), self._settings.handle, ctypes.byref(handle),
                                                      message, native._MESSAGE)
        native._raise(status, message)
        self._handle = handle

    def step(self, iterations: int = 1) -> None:
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_step(self._handle, iterations, message, self._native._MESSAGE)
        self._native._raise(status, message)

    def run(self, iterations: int, rank: int = 0, swaps: Sequence[tuple[int, int, int, int, int]] = (),
            comm: int | None = None) -> None:
        """`iterations` iterations (0: none), each followed by the exchanges of `swaps` (as
        exchanges() gives them) in which `rank` takes part, through the NCCL communicator `comm`
        (an ncclComm_t's address) on the strip's stream; not waited for."""
        table, count = _exchange_table(swaps)
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_run(self._handle, iterations, rank, table, count, comm, message,
                                                      self._native._MESSAGE)
        self._native._raise(status, message)

    def planes(self) -> list:
        """The current state's planes as device tensors that alias the solver's memory."""
        import torch

        pointers = (ctypes.POINTER(ctypes.c_float) * 64)()
        rows, columns, pitch = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        count = int(self._library.unround_b200_strip_state(self._handle, pointers, 64, ctypes.byref(rows),
                                                           ctypes.byref(columns), ctypes.byref(pitch)))
        return [torch.as_tensor(_DevicePlane(ctypes.cast(pointers[k], ctypes.c_void_p).value, rows.value,
                                             columns.value, pitch.value), device="cuda") for k in range(count)]

    def plan(self) -> StripPlan:
        values = (ctypes.c_double * 11)()
        self._library.unround_b200_strip_plan(self._handle, values, 11)
        return StripPlan.of(list(values))

    def set_rows(self, first: int, end: int) -> None:
        """The canvas rows [first, end) whose terms the strip's records count: its own bands."""
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_rows(self._handle, first, end, message, self._native._MESSAGE)
        self._native._raise(status, message)

    def record(self, advance: bool) -> list[float]:
        """One iteration keeping its tilde point (none when not `advance`: the start's), and the
        record's first sums over the strip's own rows."""
        sums = (ctypes.c_double * 5)()
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_record(self._handle, 1 if advance else 0, sums, message,
                                                         self._native._MESSAGE)
        self._native._raise(status, message)
        return list(sums)

    def record_duals(self, theta: float) -> list[float]:
        """The record's second sums at the scaling theta."""
        sums = (ctypes.c_double * 3)()
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_record_duals(self._handle, theta, sums, message,
                                                               self._native._MESSAGE)
        self._native._raise(status, message)
        return list(sums)

    def result(self, stop: int) -> object:
        """The result after the last iteration made (a Decoded of the strip's canvas)."""
        result = ctypes.c_void_p()
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_result(self._handle, stop, ctypes.byref(result), message,
                                                         self._native._MESSAGE)
        self._native._raise(status, message)
        try:
            return self._native._decoded(self._library, result, problems=False)
        finally:
            self._library.unround_result_free(result)

    def finish(self) -> object:
        """The last iteration and the result (a Decoded of the strip's canvas)."""
        result = ctypes.c_void_p()
        message = ctypes.create_string_buffer(self._native._MESSAGE)
        status = self._library.unround_b200_strip_finish(self._handle, ctypes.byref(result), message,
                                                         self._native._MESSAGE)
        self._native._raise(status, message)
        try:
            return self._native._decoded(self._library, result, problems=False)
        finally:
            self._library.unround_result_free(result)

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle:
            self._library.unround_b200_strip_free(handle)
            self._handle = None


class _Exchange(ctypes.Structure):
    _fields_ = [("sender", ctypes.c_int32), ("receiver", ctypes.c_int32), ("sender_row", ctypes.c_uint64),
                ("receiver_row", ctypes.c_uint64), ("rows", ctypes.c_uint64)]


def _exchange_table(swaps: Sequence[tuple[int, int, int, int, int]]) -> tuple[object, int]:
    table = (_Exchange * max(1, len(swaps)))()
    for k, (sender, s_row, receiver, r_row, count) in enumerate(swaps):
        table[k] = _Exchange(sender, receiver, s_row, r_row, count)
    return table, len(swaps)


def exchange_local(solvers: Sequence[StripSolver], swaps: Sequence[tuple[int, int, int, int, int]]) -> None:
    """The swaps among strips of one process (sender and receiver index `solvers`): device copies
    ordered after each sender's work so far and before its next, not waited for."""
    if not solvers:
        return
    first = solvers[0]
    handles = (ctypes.c_void_p * len(solvers))(*[s._handle.value for s in solvers])
    table, count = _exchange_table(swaps)
    message = ctypes.create_string_buffer(first._native._MESSAGE)
    status = first._library.unround_b200_strip_exchange_local(handles, len(solvers), table, count, message,
                                                              first._native._MESSAGE)
    first._native._raise(status, message)


def _bind(library: ctypes.CDLL) -> None:
    text = (ctypes.c_char_p, ctypes.c_size_t)
    u64, u64p, handle = ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p
    table = {
        "unround_b200_strip_new": (ctypes.c_int32, ctypes.c_void_p, handle, ctypes.POINTER(handle), *text),
        "unround_b200_strip_step": (ctypes.c_int32, handle, u64, *text),
        "unround_b200_strip_state": (u64, handle, ctypes.c_void_p, u64, u64p, u64p, u64p),
        "unround_b200_strip_finish": (ctypes.c_int32, handle, ctypes.POINTER(handle), *text),
        "unround_b200_strip_free": (None, handle),
        "unround_b200_strip_plan": (u64, handle, ctypes.c_void_p, u64),
        "unround_b200_strip_rows": (ctypes.c_int32, handle, u64, u64, *text),
        "unround_b200_strip_record": (ctypes.c_int32, handle, ctypes.c_int32, ctypes.c_void_p, *text),
        "unround_b200_strip_record_duals": (ctypes.c_int32, handle, ctypes.c_double, ctypes.c_void_p, *text),
        "unround_b200_strip_result": (ctypes.c_int32, handle, ctypes.c_int32, ctypes.POINTER(handle), *text),
        "unround_b200_strip_run": (ctypes.c_int32, handle, u64, ctypes.c_int32, ctypes.c_void_p, u64, ctypes.c_void_p,
                                   *text),
        "unround_b200_strip_exchange_local": (ctypes.c_int32, ctypes.c_void_p, u64, ctypes.c_void_p, u64, *text),
    }
    for name, (result, *arguments) in table.items():
        function = getattr(library, name)
        function.restype = result
        function.argtypes = arguments


@dataclass(frozen=True)
class StripPlan:
    """What of a strip's plan the driver needs: its iterations, records and stops, weights."""

    iterations: int
    record_every: int
    tolerance: float
    relative_tolerance: float
    partial_tolerance: float
    partial_radius: float | None
    alpha: float
    alpha1: float
    alpha0: float
    tgv: bool

    @staticmethod
    def of(values: Sequence[float]) -> StripPlan:
        return StripPlan(int(values[0]), int(values[1]), values[2], values[3], values[4],
                         None if math.isnan(values[5]) else values[5], values[6], values[7], values[8],
                         values[9] == 2.0)

    def recorded(self, n: int) -> bool:
        return (self.record_every > 0 and n % self.record_every == 0) or n == self.iterations


@dataclass(frozen=True)
class StripSolution:
    """A solve in strips: this rank's own rows of the canvas (all of it from solve_in_strips),
    the picture's records (native.History), its iterations and why it stopped."""

    canvas: npt.NDArray[np.float64]
    history: object
    iterations: int
    stop: int


def combine(plan: StripPlan, firsts: Sequence[Sequence[float]],
            second_of: Callable[[float], Sequence[Sequence[float]]]) -> tuple[tuple[float, ...], float]:
    """A record of the picture from every rank's sums, in rank order: `firsts` each rank's
    {G, first-order norms, second-order norms, largest |div2 r~|, samples}; `second_of(theta)`
    each rank's {conjugates, partial gap's conjugates, its residual} at theta. Returns (primal,
    dual, scaling, partial gap) and the samples, in the whole solve's binary64 arithmetic
    (cpp/src/primal_dual.hpp:446-501)."""
    data = first = second = samples = 0.0
    most = 0.0
    for f in firsts:
        data += f[0]
        first += f[1]
        second += f[2]
        most = max(most, f[3])
        samples += f[4]
    nan = float("nan")
    if not plan.tgv:
        primal = plan.alpha * first + data
        conjugates = 0.0
        for s in second_of(1.0):
            conjugates += s[0]
        return (primal, -conjugates, nan, nan), samples
    primal = (plan.alpha1 * first + plan.alpha0 * second) + data
    theta = plan.alpha1 / most if most > plan.alpha1 else 1.0
    conjugates = partial = residual = 0.0
    for s in second_of(theta):
        conjugates += s[0]
        partial += s[1]
        residual += s[2]
    partial_gap = primal + partial + plan.partial_radius * residual if plan.partial_radius is not None else nan
    return (primal, -conjugates, theta, partial_gap), samples


def _met(plan: StripPlan, values: tuple[float, ...], samples: float) -> bool:
    """Whether a record meets a tolerance of the plan (the whole solve's stops)."""
    primal, dual, _, partial_gap = values
    gap = primal - dual
    if plan.tolerance > 0.0 and gap / samples <= plan.tolerance:
        return True
    if plan.relative_tolerance > 0.0 and gap <= plan.relative_tolerance * primal:
        return True
    return plan.partial_tolerance > 0.0 and not math.isnan(partial_gap) and partial_gap / samples <= plan.partial_tolerance


def _drive(plan: StripPlan, run: Callable[[int], None], firsts_of: Callable[[bool], Sequence[Sequence[float]]],
           seconds_of: Callable[[float], Sequence[Sequence[float]]]) -> tuple[list[tuple], int, int]:
    """The method's loop over the strips, as the whole solve runs it: a record at 0 (where the plan
    records) and at every recorded iteration, each the ranks' sums combined; the halos swapped
    after the start and after every iteration; a tolerance met stops every rank there. `run(k)`
    makes k iterations, each followed by the swap (k = 0: the swap alone); the iterations between
    two records are one call. Returns the records (iteration, seconds 0, primal, dual, scaling,
    partial gap), the iterations made and the stop (1 converged, 2 iterations)."""
    records: list[tuple] = []
    run(0)  # the start's halos

    def take(iteration: int, advance: bool) -> bool:
        values, samples = combine(plan, firsts_of(advance), seconds_of)
        records.append((iteration, 0.0, *values))
        return _met(plan, values, samples)

    if (plan.record_every > 0 or plan.iterations == 0) and take(0, False):
        return records, 0, 1
    n = 0
    while n < plan.iterations:
        # The next recorded iteration (the last one always is).
        recorded = plan.iterations
        if plan.record_every > 0:
            recorded = min(plan.iterations, (n // plan.record_every + 1) * plan.record_every)
        if recorded - 1 > n:
            run(recorded - 1 - n)
        n = recorded
        met = take(n, True)
        run(0)
        if met:
            return records, n, 1
    return records, plan.iterations, 2


def _history(records: list[tuple]) -> object:
    from unround import native

    columns = list(zip(*records)) if records else [()] * 6
    arrays = [np.asarray(column, dtype=np.float64) for column in columns[1:]]
    return native.History(np.asarray(columns[0], dtype=np.int64), *arrays)


def solve_in_strips(image: jpegio.Image, options: list[str], strips: int = 2) -> StripSolution:
    """The whole solve of `image` with its bands in `strips` strips, each its own solver on the
    current device, the halo swaps device copies between them and the records the strips' sums
    added in strip order: the canvas (channels x rows x columns), the records and the stop,
    which are the whole solve's."""
    import torch

    rows = band_rows(image)
    parts = partition(band_count(image), strips)
    solvers = [StripSolver(sub_image(image, part), options) for part in parts]
    for solver, part in zip(solvers, parts):
        solver.set_rows((part.first - part.low) * rows, (part.end - part.low) * rows)
    plan = solvers[0].plan()

    swaps = exchanges(parts, rows)

    def run(count: int) -> None:
        for _ in range(count):
            for solver in solvers:
                solver.run(1)
            exchange_local(solvers, swaps)
        if count == 0:
            exchange_local(solvers, swaps)

    records, iterations, stop = _drive(plan, run, lambda advance: [s.record(advance) for s in solvers],
                                       lambda theta: [s.record_duals(theta) for s in solvers])
    decoded = [solver.result(stop) for solver in solvers]
    canvas = np.concatenate([_own_rows(d, part, rows) for d, part in zip(decoded, parts)], axis=1)
    return StripSolution(canvas, _history(records), iterations, stop)


def _gathered(values: Sequence[float], group: object) -> list[list[float]]:
    """Every rank's values, in rank order (NCCL: through the device; gloo: the host)."""
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    mine = torch.tensor(list(values), dtype=torch.float64, device=device)
    every = [torch.empty_like(mine) for _ in range(dist.get_world_size(group))]
    dist.all_gather(every, mine, group=group)
    return [t.cpu().tolist() for t in every]


def _communicator(group: object) -> int | None:
    """The address of `group`'s NCCL communicator on this rank's device (torch's
    ProcessGroupNCCL), made by a first collective; None where the backend is not NCCL or torch does
    not expose it."""
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) != "nccl":
        return None
    owner = group if group is not None else dist.distributed_c10d._get_default_group()
    try:
        dist.all_reduce(torch.zeros(1, device="cuda"), group=group)
        backend = owner._get_backend(torch.device("cuda", torch.cuda.current_device()))
        return int(backend._comm_ptr())
    except (AttributeError, RuntimeError):
        return None


def drive_rank(solver: object, parts: list[Strip], rank: int, rows: int, group: object = None) -> tuple:
    """This rank's loop over its strip's `solver` (a StripSolver, or any object with its plan,
    set_rows, step, planes, record, record_duals and result): the swaps with its neighbours and
    the records gathered from every rank. With NCCL and a StripSolver the iterations between two
    records and their swaps are one library call (StripSolver.run: NCCL sends and receives of
    torch's communicator on the strip's stream, no host wait); otherwise each iteration is a step
    and a swap through torch.distributed. Returns (the result of the strip, the records, the
    iterations made, the stop)."""
    part = parts[rank]
    solver.set_rows((part.first - part.low) * rows, (part.end - part.low) * rows)
    plan = solver.plan()
    comm = _communicator(group) if isinstance(solver, StripSolver) else None
    if comm is not None:
        swaps = exchanges(parts, rows)

        def run(count: int) -> None:
            solver.run(count, rank, swaps, comm)
    else:
        def run(count: int) -> None:
            for _ in range(count):
                solver.step(1)
                exchange(solver.planes(), parts, rank, rows, group)
            if count == 0:
                exchange(solver.planes(), parts, rank, rows, group)

    records, iterations, stop = _drive(plan, run, lambda advance: _gathered(solver.record(advance), group),
                                       lambda theta: _gathered(solver.record_duals(theta), group))
    return solver.result(stop), records, iterations, stop


def _own_rows(decoded: object, strip: Strip, rows: int) -> npt.NDArray[np.float64]:
    canvas = decoded.canvas  # type: ignore[attr-defined]
    start = (strip.first - strip.low) * rows
    return canvas[:, start : start + (strip.end - strip.first) * rows]


def solve_strip(image: jpegio.Image, options: list[str], group: object = None) -> StripSolution:
    """This rank's part of the solve of `image` in strips under torch.distributed (one rank a
    GPU, the swaps NCCL sends and receives with its neighbours, the records' sums gathered from
    every rank): the rows of the canvas it owns (channels x rows x columns), concatenated in rank
    order the whole solve's canvas, and the picture's records and stop, alike on every rank."""
    import torch.distributed as dist

    rank, ranks = dist.get_rank(group), dist.get_world_size(group)
    rows = band_rows(image)
    parts = partition(band_count(image), ranks)
    solver = StripSolver(sub_image(image, parts[rank]), options)
    decoded, records, iterations, stop = drive_rank(solver, parts, rank, rows, group)
    return StripSolution(_own_rows(decoded, parts[rank], rows), _history(records), iterations, stop)
