"""Test infrastructure: the oracle. The reference's own C++ solver, compiled in place.

oracle/ref/Makefile compiles JPEG-Unround's C++ implementation (cpp/src: dct, exact,
laplace, model, operators, frames, pdhg, settings, subgradient, colour), which the
reference checks against the same conformance cases as its Rust implementation, into
oracle/_ref/libunround_ref.so with the C face of oracle/ref/bridge.cpp. This module
loads it through ctypes. Only tests, __graft_entry__.smoke() and bench.py's CPU
baseline use it, as the checker; nothing of the product imports it.

The path followed is the reference's array-level solve: parse_settings
(cpp/src/settings.cpp:243), Frame::make (cpp/src/frames.cpp:155) and pdhg::solve
(cpp/src/pdhg.cpp:235), records at the start, every record_every iterations and at the
last (cpp/src/primal_dual.hpp:957-1013).
"""

from __future__ import annotations

import ctypes
import functools
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_ref" / "libunround_ref.so"


class _Component(ctypes.Structure):
    _fields_ = (
        ("levels", ctypes.POINTER(ctypes.c_int16)),
        ("rows", ctypes.c_uint32),
        ("columns", ctypes.c_uint32),
        ("h", ctypes.c_int32),
        ("v", ctypes.c_int32),
        ("table", ctypes.c_uint16 * 64),
    )


class _Start(ctypes.Structure):
    _fields_ = (
        ("coefficients", ctypes.POINTER(ctypes.c_double)),
        ("p", ctypes.POINTER(ctypes.c_double)),
        ("w", ctypes.POINTER(ctypes.c_double)),
        ("r", ctypes.POINTER(ctypes.c_double)),
    )


def available() -> bool:
    return LIBRARY.is_file()


@functools.cache
def _library() -> ctypes.CDLL:
    if not LIBRARY.is_file():
        raise FileNotFoundError(f"{LIBRARY} is not built: run make -C oracle/ref")
    lib = ctypes.CDLL(str(LIBRARY))
    u64p = ctypes.POINTER(ctypes.c_uint64)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.oref_solve.restype = ctypes.c_void_p
    lib.oref_solve.argtypes = (
        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint32, ctypes.POINTER(_Component),
        ctypes.c_size_t, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(_Start), ctypes.c_char_p, ctypes.c_size_t,
    )
    lib.oref_free.argtypes = (ctypes.c_void_p,)
    lib.oref_project.restype = ctypes.c_int
    lib.oref_project.argtypes = (
        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint32, ctypes.POINTER(_Component),
        ctypes.c_size_t, ctypes.POINTER(ctypes.c_char_p), dp, ctypes.c_size_t, dp, dp, dp, ctypes.c_char_p,
        ctypes.c_size_t,
    )
    lib.oref_shape.argtypes = (ctypes.c_void_p, u64p, u64p, u64p)
    lib.oref_canvas.restype = dp
    lib.oref_canvas.argtypes = (ctypes.c_void_p,)
    lib.oref_array.restype = dp
    lib.oref_array.argtypes = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32, u64p)
    lib.oref_flat.restype = ctypes.POINTER(ctypes.c_uint8)
    lib.oref_flat.argtypes = (ctypes.c_void_p, ctypes.c_uint32, u64p)
    lib.oref_component.argtypes = (ctypes.c_void_p, ctypes.c_uint32, u64p, u64p, u64p, u64p)
    lib.oref_records.restype = ctypes.c_uint64
    lib.oref_records.argtypes = (ctypes.c_void_p, ctypes.POINTER(u64p), ctypes.POINTER(dp))
    lib.oref_solver.argtypes = (ctypes.c_void_p, u64p, ctypes.POINTER(ctypes.c_int32), dp, dp)
    lib.oref_solve_samples.restype = ctypes.c_void_p
    lib.oref_solve_samples.argtypes = (
        ctypes.POINTER(ctypes.c_uint16), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32,
        ctypes.c_size_t, ctypes.POINTER(ctypes.c_char_p), ctypes.c_char_p, ctypes.c_size_t,
    )
    return lib


@dataclass
class Solved:
    """What the reference solver made: the canvas (C, H, W), each component's coefficients
    (rows, columns, 8, 8) and model, the records (iteration; seconds, primal, dual, scaling,
    partial gap), the iterations, the stop (1 converged, 2 iterations, 3 observer) and steps."""

    canvas: np.ndarray
    coefficients: list[np.ndarray]
    lower: list[np.ndarray]
    upper: list[np.ndarray]
    centres: list[np.ndarray]
    weights: list[np.ndarray]
    flat_weights: list[np.ndarray]
    flat: list[np.ndarray]
    cells: list[tuple[int, int]]
    record_iterations: np.ndarray
    records: np.ndarray
    iterations: int
    stop: int
    tau: float
    sigma: float


def solve(
    height: int,
    width: int,
    color_space: int,
    components: list[tuple[np.ndarray, np.ndarray, int, int]],
    options: list[str],
    start: dict[str, np.ndarray] | None = None,
) -> Solved:
    """Runs the reference solver. components: (levels (rows, columns, 8, 8) int16, table (64,)
    uint16 in natural order, h, v). start: optional 'coefficients' (all components' blocks one
    after another), 'p' (C, 2, H, W), 'w' (C, 2, H, W), 'r' (C, 3, H, W)."""
    lib = _library()
    kept = []
    raw = (_Component * len(components))()
    for index, (levels, table, h, v) in enumerate(components):
        levels = np.ascontiguousarray(levels, dtype=np.int16)
        kept.append(levels)
        raw[index].levels = levels.ctypes.data_as(ctypes.POINTER(ctypes.c_int16))
        raw[index].rows, raw[index].columns = levels.shape[0], levels.shape[1]
        raw[index].h, raw[index].v = h, v
        raw[index].table = (ctypes.c_uint16 * 64)(*(int(step) for step in np.asarray(table).reshape(64)))
    encoded = [option.encode() for option in options]
    array = (ctypes.c_char_p * max(len(encoded), 1))(*encoded)
    start_struct = None
    if start is not None:
        start_struct = _Start()
        for name in ("coefficients", "p", "w", "r"):
            if name in start and start[name] is not None:
                values = np.ascontiguousarray(start[name], dtype=np.float64)
                kept.append(values)
                setattr(start_struct, name, values.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    message = ctypes.create_string_buffer(4096)
    handle = lib.oref_solve(
        height, width, color_space, len(components), raw, len(encoded), array,
        ctypes.byref(start_struct) if start_struct is not None else None, message, 4096,
    )
    if not handle:
        raise ValueError(message.value.decode())
    try:
        c, h, w = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        lib.oref_shape(handle, ctypes.byref(c), ctypes.byref(h), ctypes.byref(w))
        shape = (c.value, h.value, w.value)
        canvas = np.ctypeslib.as_array(lib.oref_canvas(handle), shape=shape).copy()
        arrays: dict[int, list[np.ndarray]] = {k: [] for k in range(6)}
        flats, cells = [], []
        for index in range(c.value):
            br, bc, cr, cc = (ctypes.c_uint64() for _ in range(4))
            lib.oref_component(handle, index, ctypes.byref(br), ctypes.byref(bc), ctypes.byref(cr), ctypes.byref(cc))
            cells.append((cr.value, cc.value))
            for which in range(6):
                count = ctypes.c_uint64()
                pointer = lib.oref_array(handle, index, which, ctypes.byref(count))
                values = np.ctypeslib.as_array(pointer, shape=(count.value,)).copy() if count.value else np.zeros(0)
                arrays[which].append(values.reshape(8, 8) if which >= 4 else values.reshape(br.value, bc.value, 8, 8))
            count = ctypes.c_uint64()
            pointer = lib.oref_flat(handle, index, ctypes.byref(count))
            flats.append(np.ctypeslib.as_array(pointer, shape=(count.value,)).copy().reshape(br.value, bc.value))
        iterations_p = ctypes.POINTER(ctypes.c_uint64)()
        values_p = ctypes.POINTER(ctypes.c_double)()
        n = lib.oref_records(handle, ctypes.byref(iterations_p), ctypes.byref(values_p))
        record_iterations = np.ctypeslib.as_array(iterations_p, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
        records = np.ctypeslib.as_array(values_p, shape=(n, 5)).copy() if n else np.zeros((0, 5))
        iterations, stop = ctypes.c_uint64(), ctypes.c_int32()
        tau, sigma = ctypes.c_double(), ctypes.c_double()
        lib.oref_solver(handle, ctypes.byref(iterations), ctypes.byref(stop), ctypes.byref(tau), ctypes.byref(sigma))
        return Solved(
            canvas=canvas, coefficients=arrays[0], lower=arrays[1], upper=arrays[2], centres=arrays[3],
            weights=arrays[4], flat_weights=arrays[5], flat=flats, cells=cells,
            record_iterations=record_iterations.astype(np.int64), records=records,
            iterations=iterations.value, stop=stop.value, tau=tau.value, sigma=sigma.value,
        )
    finally:
        lib.oref_free(handle)


@dataclass
class SolvedSamples:
    """What the reference made of a picture of rounded samples: its planes (C, H, W), the
    colours' records (iteration; seconds, primal, dual, scaling, partial gap), iterations, stop
    (1 converged, 2 iterations) and steps."""

    canvas: np.ndarray
    record_iterations: np.ndarray
    records: np.ndarray
    iterations: int
    stop: int
    tau: float
    sigma: float


def solve_samples(levels: np.ndarray, bits: int, options: list[str]) -> SolvedSamples:
    """Runs the reference's solver of rounded samples (cpp/src/samples.cpp) on levels (H, W) or
    (H, W, C) of `bits` bits, as it reconstructs a PNG file's."""
    lib = _library()
    values = np.ascontiguousarray(levels, dtype=np.uint16)
    if values.ndim == 2:
        values = values[:, :, np.newaxis]
    rows, columns, channels = values.shape
    encoded = [option.encode() for option in options]
    array = (ctypes.c_char_p * max(len(encoded), 1))(*encoded)
    message = ctypes.create_string_buffer(4096)
    handle = lib.oref_solve_samples(values.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), rows, columns, channels,
                                    bits, len(encoded), array, message, 4096)
    if not handle:
        raise ValueError(message.value.decode())
    try:
        canvas = np.ctypeslib.as_array(lib.oref_canvas(handle), shape=(channels, rows, columns)).copy()
        iterations_p = ctypes.POINTER(ctypes.c_uint64)()
        values_p = ctypes.POINTER(ctypes.c_double)()
        n = lib.oref_records(handle, ctypes.byref(iterations_p), ctypes.byref(values_p))
        record_iterations = np.ctypeslib.as_array(iterations_p, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
        records = np.ctypeslib.as_array(values_p, shape=(n, 5)).copy() if n else np.zeros((0, 5))
        iterations, stop = ctypes.c_uint64(), ctypes.c_int32()
        tau, sigma = ctypes.c_double(), ctypes.c_double()
        lib.oref_solver(handle, ctypes.byref(iterations), ctypes.byref(stop), ctypes.byref(tau), ctypes.byref(sigma))
        return SolvedSamples(canvas=canvas, record_iterations=record_iterations.astype(np.int64), records=records,
                             iterations=iterations.value, stop=stop.value, tau=tau.value, sigma=sigma.value)
    finally:
        lib.oref_free(handle)


@dataclass
class Projected:
    """The reference's projection of a picture onto a file's intervals (cpp/src/picture.cpp:
    70-148): the projected canvas (C, rows, columns), each component's clipped coefficients and
    the picture's excess in steps (rows, columns, 8, 8)."""

    canvas: np.ndarray
    coefficients: list[np.ndarray]
    excess: list[np.ndarray]


def project(height: int, width: int, color_space: int, components: list[tuple[np.ndarray, np.ndarray, int, int]],
            options: list[str], picture: np.ndarray) -> Projected:
    """Runs the reference's projection of `picture` ((height, width) grey or (height, width, 3)
    RGB, binary64) onto the intervals of the components (as solve takes them)."""
    lib = _library()
    kept = []
    raw = (_Component * len(components))()
    for index, (levels, table, h, v) in enumerate(components):
        levels = np.ascontiguousarray(levels, dtype=np.int16)
        kept.append(levels)
        raw[index].levels = levels.ctypes.data_as(ctypes.POINTER(ctypes.c_int16))
        raw[index].rows, raw[index].columns = levels.shape[0], levels.shape[1]
        raw[index].h, raw[index].v = h, v
        raw[index].table = (ctypes.c_uint16 * 64)(*(int(step) for step in np.asarray(table).reshape(64)))
    encoded = [option.encode() for option in options]
    array = (ctypes.c_char_p * max(len(encoded), 1))(*encoded)
    samples = np.ascontiguousarray(picture, dtype=np.float64)
    channels = 1 if samples.ndim == 2 else samples.shape[2]
    v_max = max(v for _, _, _, v in components)
    h_max = max(h for _, _, h, _ in components)
    rows = -(-height // (8 * v_max)) * 8 * v_max
    columns = -(-width // (8 * h_max)) * 8 * h_max
    canvas = np.zeros((len(components), rows, columns))
    blocks = [np.asarray(levels).shape[:2] for levels, _, _, _ in components]
    total = sum(r * c * 64 for r, c in blocks)
    zeta, excess = np.zeros(total), np.zeros(total)
    dp = ctypes.POINTER(ctypes.c_double)
    message = ctypes.create_string_buffer(4096)
    status = lib.oref_project(height, width, color_space, len(components), raw, len(encoded), array,
                              samples.ctypes.data_as(dp), channels, canvas.ctypes.data_as(dp),
                              zeta.ctypes.data_as(dp), excess.ctypes.data_as(dp), message, 4096)
    if status != 0:
        raise ValueError(message.value.decode())
    out_z, out_e, offset = [], [], 0
    for r, c in blocks:
        n = r * c * 64
        out_z.append(zeta[offset : offset + n].reshape(r, c, 8, 8))
        out_e.append(excess[offset : offset + n].reshape(r, c, 8, 8))
        offset += n
    return Projected(canvas, out_z, out_e)
