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
  exchange         the swap over torch.distributed (NCCL for device tensors, gloo on the CPU)
  solve_in_strips  the whole solve with the strips in one process on one GPU (the ranks
                   emulated, the swaps device copies between them), for tests and one device
  solve_strip      a rank's part of it under torch.distributed (one process per GPU)
"""

from __future__ import annotations

import ctypes
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

    def planes(self) -> list:
        """The current state's planes as device tensors that alias the solver's memory."""
        import torch

        pointers = (ctypes.POINTER(ctypes.c_float) * 64)()
        rows, columns, pitch = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        count = int(self._library.unround_b200_strip_state(self._handle, pointers, 64, ctypes.byref(rows),
                                                           ctypes.byref(columns), ctypes.byref(pitch)))
        return [torch.as_tensor(_DevicePlane(ctypes.cast(pointers[k], ctypes.c_void_p).value, rows.value,
                                             columns.value, pitch.value), device="cuda") for k in range(count)]

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


def _bind(library: ctypes.CDLL) -> None:
    text = (ctypes.c_char_p, ctypes.c_size_t)
    u64, u64p, handle = ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p
    table = {
        "unround_b200_strip_new": (ctypes.c_int32, ctypes.c_void_p, handle, ctypes.POINTER(handle), *text),
        "unround_b200_strip_step": (ctypes.c_int32, handle, u64, *text),
        "unround_b200_strip_state": (u64, handle, ctypes.c_void_p, u64, u64p, u64p, u64p),
        "unround_b200_strip_finish": (ctypes.c_int32, handle, ctypes.POINTER(handle), *text),
        "unround_b200_strip_free": (None, handle),
    }
    for name, (result, *arguments) in table.items():
        function = getattr(library, name)
        function.restype = result
        function.argtypes = arguments


def _iterations(options: list[str]) -> int:
    """The options' iterations: a solve in strips is given them (it stops at its last only)."""
    for k, option in enumerate(options):
        if option == "--iterations" and k + 1 < len(options):
            return int(options[k + 1])
        if option.startswith("--iterations="):
            return int(option.split("=", 1)[1])
    raise ValueError("a solve in strips is given its --iterations")


def _own_rows(decoded: object, strip: Strip, rows: int) -> npt.NDArray[np.float64]:
    canvas = decoded.canvas  # type: ignore[attr-defined]
    start = (strip.first - strip.low) * rows
    return canvas[:, start : start + (strip.end - strip.first) * rows]


def solve_in_strips(image: jpegio.Image, options: list[str], strips: int = 2) -> npt.NDArray[np.float64]:
    """The whole solve of `image` with its bands in `strips` strips, each its own solver on the
    current device, the halo swaps device copies: the canvas (channels x rows x columns), which
    is the whole solve's. The options record at the last iteration only."""
    import torch

    rows = band_rows(image)
    parts = partition(band_count(image), strips)
    solvers = [StripSolver(sub_image(image, part), options) for part in parts]
    iterations = _iterations(options)

    def swap() -> None:
        planes = [solver.planes() for solver in solvers]
        torch.cuda.synchronize()
        for sender, s_row, receiver, r_row, count in exchanges(parts, rows):
            for source, target in zip(planes[sender], planes[receiver]):
                target[r_row : r_row + count].copy_(source[s_row : s_row + count])
        torch.cuda.synchronize()

    swap()  # the start's halos
    for _ in range(max(0, iterations - 1)):
        for solver in solvers:
            solver.step(1)
        swap()
    decoded = [solver.finish() for solver in solvers]
    return np.concatenate([_own_rows(d, part, rows) for d, part in zip(decoded, parts)], axis=1)


def solve_strip(image: jpegio.Image, options: list[str], group: object = None) -> npt.NDArray[np.float64]:
    """This rank's part of the solve of `image` in strips under torch.distributed (one rank a
    GPU, the swaps NCCL sends and receives with its neighbours): the rows of the canvas it owns
    (channels x rows x columns). Concatenated in rank order, they are the whole solve's canvas."""
    import torch.distributed as dist

    rank, ranks = dist.get_rank(group), dist.get_world_size(group)
    rows = band_rows(image)
    parts = partition(band_count(image), ranks)
    solver = StripSolver(sub_image(image, parts[rank]), options)
    exchange(solver.planes(), parts, rank, rows, group)
    for _ in range(max(0, _iterations(options) - 1)):
        solver.step(1)
        exchange(solver.planes(), parts, rank, rows, group)
    return _own_rows(solver.finish(), parts[rank], rows)
