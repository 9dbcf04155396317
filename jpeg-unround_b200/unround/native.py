"""The reconstruction on a B200, through the C interface of libunround_capi.so.

The drop-in for the reference package's unround.native (python/src/unround/native.py of
JPEG-Unround): the same functions, data classes and errors, over the same C interface
(include/unround.h, ABI version 5), so a caller switches by importing this package. ctypes
releases the GIL while the library computes; every call has its own CUDA stream, so threads
reconstruct at once. The settings go over as the command line's options, each number as the
shortest decimal that reads back as the same double (repr); the results come back as NumPy
arrays, copied, and the library's memory is freed before a function returns.

solve() is the path: levels and tables in, the TV/TGV primal-dual solve on the GPU, the
binary64 result out. decode() reads a JPEG file's coefficients (or a PNG file's levels) on the
host with this build's own readers and solves them the same way; project() measures a picture
against a file's intervals on the host. solve_from(), measure(), solve_batch() and the other
functions without a counterpart in the reference are this build's extensions
(include/unround_b200.h).

The library is the file that the environment variable UNROUND_LIBRARY names, where it is set,
as the reference's package looks it up; otherwise libunround_capi.so in this package's _native
folder, where jpeg-unround_b200/build.py writes it.
"""

from __future__ import annotations

import ctypes
import enum
import functools
import os
import threading
import warnings
from collections.abc import Callable
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from pathlib import Path
from typing import Final

import numpy as np
import numpy.typing as npt

from unround import jpegio
from unround.settings import TGV, TV, DataTerm, PdhgOptions, Settings, SubgradientOptions

__all__ = [
    "ABI_VERSION",
    "BatchTiming",
    "Decoded",
    "History",
    "LibraryNotFoundError",
    "Problem",
    "Record",
    "Solution",
    "Status",
    "Stop",
    "Timing",
    "UnroundError",
    "UnroundWarning",
    "decode",
    "held_options",
    "library_path",
    "measure",
    "model",
    "options",
    "project",
    "solve",
    "solve_batch",
    "solve_from",
    "to_rgb",
    "to_ycbcr",
    "version",
]

type Array = npt.NDArray[np.float64]
type Observer = Callable[["Record"], bool | None]

ABI_VERSION: Final = 5
_MESSAGE: Final = 4096


class _Record(ctypes.Structure):
    _fields_ = (
        ("iteration", ctypes.c_uint64),
        ("gap", ctypes.c_double),
        ("primal", ctypes.c_double),
        ("dual", ctypes.c_double),
        ("channels", ctypes.c_uint64),
        ("height", ctypes.c_uint64),
        ("width", ctypes.c_uint64),
        ("canvas", ctypes.POINTER(ctypes.c_double)),
    )


class _Component(ctypes.Structure):
    _fields_ = (
        ("levels", ctypes.POINTER(ctypes.c_int16)),
        ("rows", ctypes.c_uint32),
        ("columns", ctypes.c_uint32),
        ("h_samp_factor", ctypes.c_int32),
        ("v_samp_factor", ctypes.c_int32),
        ("quant_table", ctypes.c_uint16 * 64),
    )


class _Input(ctypes.Structure):
    _fields_ = (
        ("height", ctypes.c_uint32),
        ("width", ctypes.c_uint32),
        ("color_space", ctypes.c_int32),
        ("count", ctypes.c_uint32),
        ("components", ctypes.POINTER(_Component)),
    )


class _Start(ctypes.Structure):
    _fields_ = (
        ("coefficients", ctypes.POINTER(ctypes.c_double)),
        ("p", ctypes.POINTER(ctypes.c_double)),
        ("w", ctypes.POINTER(ctypes.c_double)),
        ("r", ctypes.POINTER(ctypes.c_double)),
    )


class _Timing(ctypes.Structure):
    _fields_ = (
        ("milliseconds", ctypes.c_double),
        ("dual_milliseconds", ctypes.c_double),
        ("primal_milliseconds", ctypes.c_double),
        ("iterations", ctypes.c_uint64),
        ("launches_per_iteration", ctypes.c_uint64),
        ("samples", ctypes.c_uint64),
        ("pixels", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
    )


class _BatchTiming(ctypes.Structure):
    _fields_ = (
        ("milliseconds", ctypes.c_double),
        ("iterations", ctypes.c_uint64),
        ("launches_per_iteration", ctypes.c_uint64),
        ("samples", ctypes.c_uint64),
        ("pixels", ctypes.c_uint64),
        ("tuning_milliseconds", ctypes.c_double),
    )


_SIZES: Final = ((_Record, 64), (_Component, 152), (_Input, 24))
_OBSERVER: Final = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(_Record))


class Status(enum.IntEnum):
    """unround_status."""

    OK = 0
    ARGUMENT = 1
    READ = 2
    UNSUPPORTED = 3
    OPTIONS = 4
    IO = 5
    INTERNAL = 6


class Stop(enum.IntEnum):
    """Why a solver stopped."""

    CONVERGED = 1
    ITERATIONS = 2
    OBSERVER = 3
    STATIONARY = 4


class UnroundError(Exception):
    """Arrays or a file that were not reconstructed: the interface's status and message."""

    def __init__(self, status: Status, message: str) -> None:
        super().__init__(f"{message} ({status.name.lower()})")
        self.status = status
        self.message = message

    def __reduce__(self) -> tuple[type[UnroundError], tuple[Status, str]]:
        return (type(self), (self.status, self.message))


class LibraryNotFoundError(RuntimeError):
    """The library is not where this module looks for it, or not of its ABI version."""


class UnroundWarning(UserWarning):
    """What a writer left out of a file."""


def _bind(library: ctypes.CDLL) -> None:
    size, handle, u64, i32 = ctypes.c_size_t, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32
    doubles, u64p, i32p = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(u64), ctypes.POINTER(i32)
    text = (ctypes.c_char_p, size)
    made = (_OBSERVER, handle, ctypes.POINTER(handle), *text)
    table = {
        "unround_abi_version": (i32,),
        "unround_version": (ctypes.c_char_p,),
        "unround_settings_new": (handle, size, ctypes.POINTER(ctypes.c_char_p), *text),
        "unround_settings_free": (None, handle),
        "unround_settings_options": (size, handle, ctypes.c_char_p, size),
        "unround_decode": (i32, ctypes.c_char_p, size, handle, *made),
        "unround_solve": (i32, ctypes.POINTER(_Input), handle, *made),
        "unround_project": (i32, ctypes.c_char_p, size, handle, doubles, u64, u64, u64, *made[2:]),
        "unround_result_free": (None, handle),
        "unround_result_picture": (doubles, handle, u64p, u64p, u64p),
        "unround_result_planes": (doubles, handle, u64p),
        "unround_result_color_space": (i32, handle),
        "unround_result_canvas": (doubles, handle, u64p, u64p, u64p),
        "unround_result_components": (u64, handle),
        "unround_result_coefficients": (doubles, handle, u64, u64p),
        "unround_result_problem": (doubles, handle, u64, i32, u64p),
        "unround_result_component": (i32, handle, u64, u64p, u64p, u64p, u64p),
        "unround_result_solver": (i32, handle, u64p, i32p),
        "unround_result_record_iterations": (u64p, handle, u64p),
        "unround_result_record_values": (doubles, handle, i32, u64p),
        "unround_to_rgb": (i32, doubles, u64, u64, doubles),
        "unround_to_ycbcr": (i32, doubles, u64, u64, doubles),
        "unround_pnm": (i32, doubles, u64, u64, u64, i32, i32, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)), u64p,
                        *text),
        "unround_bytes_free": (None, ctypes.POINTER(ctypes.c_uint8), u64),
        "unround_png": (i32, doubles, u64, u64, u64, i32, i32, i32, ctypes.POINTER(ctypes.c_uint8), u64,
                        ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)), u64p, *text),
        "unround_orient": (i32, doubles, u64, u64, u64, i32, doubles, u64p, u64p, *text),
        "unround_tiff": (i32, doubles, u64, u64, u64, i32, ctypes.POINTER(ctypes.c_uint8), u64,
                         ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)), u64p, *text),
        "unround_main": (i32, size, ctypes.POINTER(ctypes.c_char_p)),
        "unround_result_icc_profile": (ctypes.POINTER(ctypes.c_uint8), handle, u64p),
        "unround_result_exif_orientation": (i32, handle),
        "unround_result_format": (i32, handle),
        "unround_result_bits": (i32, handle),
        "unround_result_warning": (ctypes.c_char_p, handle),
        "unround_result_excess": (doubles, handle, u64, u64p),
        "unround_b200_solve_levels": (i32, ctypes.POINTER(_Input), handle, i32, i32, ctypes.c_void_p, u64, u64p,
                                      *text),
        "unround_b200_solve_samples": (i32, ctypes.POINTER(ctypes.c_uint16), u64, u64, u64, i32, handle, *made),
        "unround_b200_measure_samples": (i32, ctypes.POINTER(ctypes.c_uint16), u64, u64, u64, i32, handle, u64, u64,
                                         ctypes.POINTER(_Timing), *text),
        "unround_b200_solve_from": (i32, ctypes.POINTER(_Input), handle, ctypes.POINTER(_Start), *made),
        "unround_b200_measure": (i32, ctypes.POINTER(_Input), handle, u64, u64, ctypes.POINTER(_Timing),
                                 ctypes.POINTER(handle), *text),
        "unround_b200_model": (i32, ctypes.POINTER(_Input), handle, u64, i32, doubles, u64, u64p, *text),
        "unround_b200_solve_batch": (i32, u64, ctypes.POINTER(_Input), ctypes.POINTER(handle), ctypes.POINTER(handle),
                                     ctypes.POINTER(_BatchTiming), *text),
    }
    for name, (result, *arguments) in table.items():
        function = getattr(library, name)
        function.restype = result
        function.argtypes = arguments


def library_path() -> str:
    """The path of the library this module loads."""
    named = os.environ.get("UNROUND_LIBRARY")
    if named:
        path: Path | None = Path(named)
    else:
        built = Path(__file__).parent / "_native" / "libunround_capi.so"
        path = built if built.is_file() else None
    if path is None or not path.is_file():
        where = f"UNROUND_LIBRARY names {path}, where there is no file" if path else "the package holds no library"
        raise LibraryNotFoundError(f"{where}: build it with python jpeg-unround_b200/build.py")
    return str(path)


@functools.cache
def _library() -> ctypes.CDLL:
    for structure, size in _SIZES:
        if ctypes.sizeof(structure) != size:
            raise RuntimeError(f"{structure.__name__} is {ctypes.sizeof(structure)} bytes, not {size}")
    path = library_path()
    library = ctypes.CDLL(path)
    _bind(library)
    found = int(library.unround_abi_version())
    if found != ABI_VERSION:
        raise LibraryNotFoundError(f"{path} is of ABI version {found}, and this module of version {ABI_VERSION}")
    return library


def version() -> str:
    """The version of JPEG-Unround and the implementation, as the library says them."""
    return _library().unround_version().decode()


def _number(value: float) -> str:
    return repr(float(value))


def _data_options(data: DataTerm | tuple[DataTerm, ...]) -> list[str]:
    terms = (data,) if isinstance(data, DataTerm) else tuple(data)
    fields: tuple[tuple[str, Callable[[DataTerm], str]], ...] = (
        ("--mu", lambda t: "rule" if t.mu is None else _number(t.mu)),
        ("--mu-scale", lambda t: _number(t.mu_scale)),
        ("--mu-power", lambda t: _number(t.mu_power)),
        ("--mu-chroma", lambda t: _number(t.mu_chroma)),
        ("--weight-power", lambda t: _number(t.power)),
        ("--dc-weight", lambda t: _number(t.dc_weight)),
        ("--centres", lambda t: t.centres),
        ("--slack", lambda t: _number(t.slack)),
        ("--slack-cost", lambda t: _number(t.slack_cost)),
        ("--flat-weight", lambda t: _number(t.flat_weight)),
        ("--flat-levels", lambda t: str(t.flat_levels)),
        ("--flat-dc", lambda t: "any" if t.flat_dc is None else str(t.flat_dc)),
    )
    out: list[str] = []
    for name, of in fields:
        values = [of(term) for term in terms]
        out += [name, values[0] if len(set(values)) == 1 else ",".join(values)]
    return out


def _pdhg_options(o: PdhgOptions) -> list[str]:
    out = ["--relative-tolerance", _number(o.relative_tolerance), "--partial-tolerance", _number(o.partial_tolerance),
           "--step-product", _number(o.step_product), "--record-every", str(o.record_every),
           "--free-radius", _number(o.free_radius), "--threads", str(o.threads)]
    if o.iterations is not None:
        out += ["--iterations", str(o.iterations)]
    for name, value in (("--tolerance", o.tolerance), ("--step-ratio", o.step_ratio), ("--relaxation", o.relaxation),
                        ("--norm-squared", o.norm_squared), ("--partial-radius", o.partial_radius)):
        if value is not None:
            out += [name, _number(value)]
    if not o.scale_with_weight:
        out.append("--no-weight-scaling")
    return out


def _subgradient_options(o: SubgradientOptions) -> list[str]:
    out = ["--subgradient-iterations", str(o.iterations), "--subgradient-record-every", str(o.record_every),
           "--subgradient-step", _number(o.step), "--subgradient-decay", _number(o.decay)]
    if not o.momentum:
        out.append("--no-momentum")
    return out


def options(settings: Settings | None = None, *, max_pixels: int = 0, max_scans: int = 0,
            warnings_are_errors: bool = False) -> list[str]:
    """The command line's options that are the settings (docs/cli.md). The channel weights and
    their coupling are those of the method's model: TGV's for TGV, TV's otherwise."""
    settings = Settings() if settings is None else settings
    weights: TV | TGV = settings.tgv if settings.method == "tgv" else settings.tv
    out = ["--method", settings.method, "--alpha", _number(settings.tv.alpha),
           "--alpha1", _number(settings.tgv.alpha1), "--alpha0", _number(settings.tgv.alpha0)]
    if weights.channel_weights is not None:
        out += ["--channel-weights", ",".join(_number(w) for w in weights.channel_weights)]
    out += ["--channels", "coupled" if weights.coupled else "apart"]
    out += _data_options(settings.data) + _pdhg_options(settings.pdhg) + _subgradient_options(settings.subgradient)
    if max_pixels < 0 or max_scans < 0:
        raise ValueError(f"the limits of reading are at least 0, not {max_pixels} pixels and {max_scans} scans")
    if max_pixels:
        out += ["--max-pixels", str(max_pixels)]
    if max_scans:
        out += ["--max-scans", str(max_scans)]
    if warnings_are_errors:
        out.append("--warnings-are-errors")
    return out


class _Settings:
    """Settings of the interface made from options, freed with the object."""

    def __init__(self, given: list[str]) -> None:
        self._library = _library()
        encoded = [option.encode("utf-8") for option in given]
        array = (ctypes.c_char_p * max(len(encoded), 1))(*encoded)
        message = ctypes.create_string_buffer(_MESSAGE)
        self.handle: int | None = self._library.unround_settings_new(len(encoded), array, message, _MESSAGE)
        if not self.handle:
            raise UnroundError(Status.OPTIONS, message.value.decode("utf-8", "replace"))

    def __del__(self) -> None:
        handle = getattr(self, "handle", None)
        if handle:
            self._library.unround_settings_free(handle)
            self.handle = None


def _settings_of(settings: Settings | list[str] | None) -> _Settings:
    return _Settings(list(settings) if isinstance(settings, list) else options(settings))


def held_options(settings: Settings | list[str] | None = None, **limits: int | bool) -> list[str]:
    """The settings as the library holds them: every value as --name=value or --flag."""
    library = _library()
    handle = _Settings(list(settings) if isinstance(settings, list) else options(settings, **limits))  # type: ignore[arg-type]
    length = int(library.unround_settings_options(handle.handle, None, 0))
    buffer = ctypes.create_string_buffer(length + 1)
    library.unround_settings_options(handle.handle, buffer, length + 1)
    return buffer.value.decode("ascii").split(" ")


@dataclass(frozen=True, slots=True, eq=False)
class Record:
    """A record as an observer sees it: gap per sample, primal and dual values, canvas (C, H, W)."""

    iteration: int
    gap: float
    primal: float
    dual: float
    canvas: Array


@dataclass(frozen=True, slots=True, eq=False)
class Problem:
    """A component's model: the ratio of canvas samples per component sample, the intervals and
    centres (rows, columns, 8, 8), the steps and weights (8, 8)."""

    ratio: tuple[int, int]
    lower: Array
    upper: Array
    centres: Array
    steps: Array
    weights: Array


@dataclass(frozen=True, slots=True, eq=False)
class History:
    """The records: iterations, seconds, primal and dual values, TGV's scaling and partial gap."""

    iterations: npt.NDArray[np.int64]
    seconds: Array
    primal: Array
    dual: Array
    scaling: Array
    partial_gap: Array

    @property
    def gap(self) -> Array:
        return np.asarray(self.primal - self.dual, dtype=np.float64)


@dataclass(frozen=True, slots=True, eq=False)
class Solution:
    """What the solver did: its iterations, why it stopped, and its records."""

    iterations: int
    stop: Stop
    history: History

    @property
    def converged(self) -> bool:
        return self.stop is Stop.CONVERGED


@dataclass(frozen=True, slots=True, eq=False)
class Decoded:
    """A reconstruction: the picture (H, W) or (H, W, C) in binary64, the planes (C, H, W), the
    canvas (C, canvas rows, canvas columns), each component's coefficients and model, and the
    solver's result (None for the decoder of the centres)."""

    picture: Array
    planes: Array
    canvas: Array
    color_space: jpegio.ColorSpace
    coefficients: tuple[Array, ...]
    problems: tuple[Problem, ...]
    result: Solution | None
    icc_profile: bytes | None
    exif_orientation: int
    input_format: str = "jpeg"
    bits: int = 8
    alpha_result: Solution | None = None
    excess: tuple[Array, ...] | None = None


# A result's large arrays are copied out of the library's memory in parts on the host's threads
# (NumPy copies without holding the interpreter): a 4032x3024 colour solve's result and model
# are about 1.3 GB, which one thread copies in ~0.4 s.
_PARALLEL_BYTES: Final = 16 << 20
_copier_lock = threading.Lock()
_copier_state: dict[str, object] = {}


def _copier() -> tuple[ThreadPoolExecutor, int]:
    with _copier_lock:
        # Made again in a child process after fork (the parent's threads do not exist there).
        if _copier_state.get("pid") != os.getpid():
            workers = max(1, min(8, os.cpu_count() or 1))
            _copier_state.update(pid=os.getpid(), workers=workers,
                                 pool=ThreadPoolExecutor(max_workers=workers, thread_name_prefix="unround-copy"))
        return _copier_state["pool"], _copier_state["workers"]  # type: ignore[return-value]


def _copy(pointer: object, shape: tuple[int, ...], dtype: type = np.float64) -> npt.NDArray:
    count = int(np.prod(shape, dtype=np.int64))
    if count == 0:
        return np.zeros(shape, dtype=dtype)
    if not pointer:
        raise RuntimeError("the library gave no values where it has some")
    source = np.ctypeslib.as_array(pointer, shape=(count,))
    if source.dtype != np.dtype(dtype) or source.nbytes < _PARALLEL_BYTES:
        return np.array(source, dtype=dtype, copy=True).reshape(shape)
    out = np.empty(count, dtype=dtype)
    pool, parts = _copier()
    step = -(-count // parts)
    list(pool.map(lambda k: np.copyto(out[k * step:(k + 1) * step], source[k * step:(k + 1) * step]), range(parts)))
    return out.reshape(shape)


def _decoded(library: ctypes.CDLL, result: ctypes.c_void_p, problems: bool = True) -> Decoded:
    u = [ctypes.c_uint64() for _ in range(4)]
    pointer = library.unround_result_picture(result, *(ctypes.byref(x) for x in u[:3]))
    rows, columns, depth = (int(x.value) for x in u[:3])
    picture = _copy(pointer, (rows, columns) if depth == 1 else (rows, columns, depth))
    pointer = library.unround_result_canvas(result, *(ctypes.byref(x) for x in u[:3]))
    channels, height, width = (int(x.value) for x in u[:3])
    canvas = _copy(pointer, (channels, height, width))
    count = ctypes.c_uint64()
    planes = _copy(library.unround_result_planes(result, ctypes.byref(count)), (channels, rows, columns))
    coefficients, models = [], []
    for index in range(int(library.unround_result_components(result))):
        library.unround_result_component(result, index, *(ctypes.byref(x) for x in u))
        block_rows, block_columns, down, across = (int(x.value) for x in u)
        shape = (block_rows, block_columns, 8, 8)
        coefficients.append(_copy(library.unround_result_coefficients(result, index, ctypes.byref(count)), shape))
        if problems:
            arrays = [_copy(library.unround_result_problem(result, index, which, ctypes.byref(count)),
                            shape if which < 3 else (8, 8)) for which in range(5)]
            models.append(Problem((down, across), *arrays))
    iterations, stop = ctypes.c_uint64(), ctypes.c_int32()
    solution = None
    if library.unround_result_solver(result, ctypes.byref(iterations), ctypes.byref(stop)):
        n = ctypes.c_uint64()
        at = library.unround_result_record_iterations(result, ctypes.byref(n))
        steps = _copy(at, (int(n.value),), np.int64)
        values = [_copy(library.unround_result_record_values(result, which, ctypes.byref(n)), (int(n.value),))
                  for which in range(5)]
        solution = Solution(int(iterations.value), Stop(int(stop.value)), History(steps, *values))
    excess = []
    for index in range(len(coefficients)):
        pointer = library.unround_result_excess(result, index, ctypes.byref(count))
        if not pointer:
            break
        excess.append(_copy(pointer, coefficients[index].shape))
    icc_size = ctypes.c_uint64()
    icc = library.unround_result_icc_profile(result, ctypes.byref(icc_size))
    return Decoded(
        picture=picture, planes=planes, canvas=canvas,
        color_space=jpegio.ColorSpace(int(library.unround_result_color_space(result))),
        coefficients=tuple(coefficients), problems=tuple(models), result=solution,
        icc_profile=ctypes.string_at(icc, int(icc_size.value)) if icc and icc_size.value else None,
        exif_orientation=int(library.unround_result_exif_orientation(result)),
        input_format="png" if int(library.unround_result_format(result)) == 2 else "jpeg",
        bits=int(library.unround_result_bits(result)),
        excess=tuple(excess) if excess else None,
    )


class _Watcher:
    """The observer as the interface calls it; an exception is kept and raised after the call."""

    def __init__(self, observer: Observer | None) -> None:
        self._observer = observer
        self.error: BaseException | None = None
        self.callback = _OBSERVER() if observer is None else _OBSERVER(self._call)

    def _call(self, _user: int | None, pointer: ctypes._Pointer[_Record]) -> int:
        if self._observer is None or self.error is not None:
            return 1
        try:
            r = pointer.contents
            seen = Record(int(r.iteration), float(r.gap), float(r.primal), float(r.dual),
                          _copy(r.canvas, (int(r.channels), int(r.height), int(r.width))))
            return 1 if self._observer(seen) else 0
        except BaseException as error:  # noqa: BLE001 -- raised again once the library returns
            self.error = error
            return 1


def _raise(status: int, message: ctypes.Array[ctypes.c_char]) -> None:
    if status != Status.OK:
        known = status in Status.__members__.values()
        raise UnroundError(Status(status) if known else Status.INTERNAL, message.value.decode("utf-8", "replace"))


def _input_of(image: jpegio.Image) -> tuple[_Input, list[object]]:
    count = len(image.components)
    kept: list[object] = []
    raw = (_Component * max(count, 1))()
    for index, component in enumerate(image.components):
        levels = np.ascontiguousarray(component.coefficients, dtype=np.int16)
        if levels.ndim != 4 or levels.shape[2:] != (8, 8):
            raise ValueError(f"the levels of component {index} are (rows, columns, 8, 8), not {levels.shape}")
        kept.append(levels)
        raw[index].levels = levels.ctypes.data_as(ctypes.POINTER(ctypes.c_int16))
        raw[index].rows, raw[index].columns = int(levels.shape[0]), int(levels.shape[1])
        raw[index].h_samp_factor = int(component.h_samp_factor)
        raw[index].v_samp_factor = int(component.v_samp_factor)
        table = np.asarray(component.quant_table, dtype=np.uint16).reshape(64)
        raw[index].quant_table = (ctypes.c_uint16 * 64)(*(int(step) for step in table))
    kept.append(raw)
    return _Input(int(image.height), int(image.width), int(image.color_space), count, raw), kept


def solve(image: jpegio.Image, settings: Settings | list[str] | None = None, *,
          observer: Observer | None = None) -> Decoded:
    """Reconstructs an image's components (levels, tables, sampling factors) on the GPU, as the
    reference's unround.native.solve does (python/src/unround/native.py:758-788). settings may
    also be the command line's options as a list of strings."""
    return solve_from(image, settings, observer=observer)


def solve_from(image: jpegio.Image, settings: Settings | list[str] | None = None, *,
               start: dict[str, npt.ArrayLike] | None = None, observer: Observer | None = None) -> Decoded:
    """solve() from a given start (include/unround_b200.h): 'coefficients' (every component's
    blocks one after another), 'p' (C, 2, H, W), 'w' (C, 2, H, W), 'r' (C, 3, H, W)."""
    library = _library()
    handle = _settings_of(settings)
    given, kept = _input_of(image)
    watcher = _Watcher(observer)
    result = ctypes.c_void_p()
    message = ctypes.create_string_buffer(_MESSAGE)
    if start is None:
        status = library.unround_solve(ctypes.byref(given), handle.handle, watcher.callback, None,
                                       ctypes.byref(result), message, _MESSAGE)
    else:
        raw = _Start()
        for name in ("coefficients", "p", "w", "r"):
            if start.get(name) is not None:
                values = np.ascontiguousarray(start[name], dtype=np.float64).reshape(-1)
                kept.append(values)
                setattr(raw, name, values.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        status = library.unround_b200_solve_from(ctypes.byref(given), handle.handle, ctypes.byref(raw),
                                                 watcher.callback, None, ctypes.byref(result), message, _MESSAGE)
    try:
        if watcher.error is not None:
            raise watcher.error
        _raise(status, message)
        return _decoded(library, result)
    finally:
        library.unround_result_free(result)
        del kept


@dataclass(frozen=True, slots=True)
class Timing:
    """measure(): the device milliseconds of the timed iterations (CUDA events), each kernel
    group's average per iteration (dual step; primal steps of every component), the iterations,
    the kernels launched per iteration, the canvas's samples and pixels, the device bytes held."""

    milliseconds: float
    dual_milliseconds: float
    primal_milliseconds: float
    iterations: int
    launches_per_iteration: int
    samples: int
    pixels: int
    device_bytes: int


def measure(image: jpegio.Image, settings: Settings | list[str] | None = None, *, warmup: int = 3,
            iterations: int = 10, result: bool = False) -> tuple[Timing, Decoded | None]:
    """Times the iteration loop alone on the GPU (include/unround_b200.h, unround_b200_measure)."""
    library = _library()
    handle = _settings_of(settings)
    given, kept = _input_of(image)
    timing = _Timing()
    made = ctypes.c_void_p()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_b200_measure(ctypes.byref(given), handle.handle, warmup, iterations,
                                          ctypes.byref(timing), ctypes.byref(made) if result else None,
                                          message, _MESSAGE)
    try:
        _raise(status, message)
        decoded = _decoded(library, made, problems=False) if result else None
        return Timing(timing.milliseconds, timing.dual_milliseconds, timing.primal_milliseconds, int(timing.iterations), int(timing.launches_per_iteration),
                      int(timing.samples), int(timing.pixels), int(timing.device_bytes)), decoded
    finally:
        if result:
            library.unround_result_free(made)
        del kept


@dataclass(frozen=True, slots=True)
class BatchTiming:
    """solve_batch(): the device milliseconds of the batched iterations (CUDA events), their
    count, the launches an iteration of the whole batch takes, and all pictures' samples and
    pixels; and the milliseconds the autotuner measured the tile heights for, before them."""

    milliseconds: float
    iterations: int
    launches_per_iteration: int
    samples: int
    pixels: int
    tuning_milliseconds: float = 0.0


def solve_batch(images: list[jpegio.Image], settings: Settings | list[str] | list | None = None
                ) -> tuple[list[Decoded], BatchTiming]:
    """Solves many pictures together on the GPU (include/unround_b200.h, unround_b200_solve_batch):
    each result is the one solve() gives that picture alone. settings: one for all pictures, or
    a list with one per picture (Settings or option lists); all take tv or tgv, the same number
    of iterations and --record-every 0."""
    library = _library()
    count = len(images)
    if count == 0:
        raise ValueError("a batch has at least one picture")
    per_picture = isinstance(settings, list) and len(settings) == count and not all(
        isinstance(s, str) for s in settings)
    handles = [_settings_of(settings[n] if per_picture else settings) for n in range(count)]
    inputs = (_Input * count)()
    kept: list[object] = []
    for n, image in enumerate(images):
        given, held = _input_of(image)
        inputs[n] = given
        kept.append(held)
    settings_array = (ctypes.c_void_p * count)(*(h.handle for h in handles))
    results = (ctypes.c_void_p * count)()
    timing = _BatchTiming()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_b200_solve_batch(count, inputs, settings_array, results, ctypes.byref(timing), message,
                                              _MESSAGE)
    try:
        _raise(status, message)
        decoded = [_decoded(library, results[n]) for n in range(count)]
        return decoded, BatchTiming(timing.milliseconds, int(timing.iterations), int(timing.launches_per_iteration),
                                    int(timing.samples), int(timing.pixels), float(timing.tuning_milliseconds))
    finally:
        for n in range(count):
            if results[n]:
                library.unround_result_free(results[n])
        del kept


def model(image: jpegio.Image, settings: Settings | list[str] | None = None, component: int = 0,
          which: int = 0) -> npt.NDArray[np.float64]:
    """What the host model makes of the input, without a GPU (include/unround_b200.h,
    unround_b200_model): which 0/1/2 the intervals' ends and centres, 3/4/5 steps, weights and
    flat blocks' weights, 6 the flat blocks, 7 the plan (tau, sigma, iterations, tolerance)."""
    library = _library()
    handle = _settings_of(settings)
    given, kept = _input_of(image)
    count = ctypes.c_uint64()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_b200_model(ctypes.byref(given), handle.handle, component, which, None, 0,
                                        ctypes.byref(count), message, _MESSAGE)
    _raise(status, message)
    out = np.empty(int(count.value))
    status = library.unround_b200_model(ctypes.byref(given), handle.handle, component, which,
                                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size,
                                        ctypes.byref(count), message, _MESSAGE)
    _raise(status, message)
    del kept
    return out


def decode(source: object, settings: Settings | list[str] | None = None, *, observer: Observer | None = None,
           max_pixels: int = 0, max_scans: int = 0, warnings_are_errors: bool = False) -> Decoded:
    """Reconstructs a JPEG file or a PNG file: its bytes or its path; or a JPEG file's components as
    unround.jpegio.read gives them (rust/capi/src/lib.rs, unround_decode).

    A PNG file, known by its signature, is reconstructed within the intervals of its rounded
    samples by TV or TGV, its colours together and its alpha alone; any other file as a JPEG file,
    its coefficients read on the host and the iterations run on the GPU. The limits of reading are
    those of unround.jpegio.read (a PNG file takes max_pixels alone). A warning of the reading (a
    JPEG file's corrupt data, a PNG file's transparent colour that is not taken) is said as an
    UnroundWarning; a file that is not reconstructed raises UnroundError."""
    if isinstance(source, jpegio.Image):
        if max_pixels or max_scans or warnings_are_errors:
            raise ValueError("an image read already takes no limits of reading")
        return solve(source, settings, observer=observer)
    if isinstance(settings, list):
        given = list(settings)
        if max_pixels:
            given += ["--max-pixels", str(max_pixels)]
        if max_scans:
            given += ["--max-scans", str(max_scans)]
        if warnings_are_errors:
            given.append("--warnings-are-errors")
    else:
        given = options(settings, max_pixels=max_pixels, max_scans=max_scans, warnings_are_errors=warnings_are_errors)
    library = _library()
    handle = _Settings(given)
    data = Path(source).read_bytes() if isinstance(source, (str, os.PathLike)) else bytes(source)  # type: ignore[arg-type]
    watcher = _Watcher(observer)
    result = ctypes.c_void_p()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_decode(data, len(data), handle.handle, watcher.callback, None, ctypes.byref(result),
                                    message, _MESSAGE)
    if watcher.error is not None:
        if status == 0:
            library.unround_result_free(result)
        raise watcher.error
    _raise(status, message)
    try:
        warning = library.unround_result_warning(result)
        if warning:
            warnings.warn(warning.decode("utf-8", "replace"), UnroundWarning, stacklevel=2)
        return _decoded(library, result, problems=int(library.unround_result_format(result)) != 2)
    finally:
        library.unround_result_free(result)


def project(picture: npt.ArrayLike, source: object, settings: Settings | list[str] | None = None, *,
            max_pixels: int = 0, max_scans: int = 0, warnings_are_errors: bool = False) -> Decoded:
    """Measures a picture against a JPEG file's intervals and projects it onto them
    (unround_project; docs/math.md 12 of the reference). picture is of the file's size as the file
    stores it, before its EXIF orientation: (height, width) of a greyscale file, or (height,
    width, 3) of RGB of a file in colour, made elsewhere, by another decoder, say; source is the
    file's bytes or path. The result is the projection, as a reconstruction without a solver
    (result is None), and its excess holds the picture's: how far each coefficient lay outside its
    interval, in steps. A picture of another size or of other channels raises UnroundError."""
    if isinstance(settings, list):
        given = list(settings)
        if max_pixels:
            given += ["--max-pixels", str(max_pixels)]
        if max_scans:
            given += ["--max-scans", str(max_scans)]
        if warnings_are_errors:
            given.append("--warnings-are-errors")
    else:
        given = options(settings, max_pixels=max_pixels, max_scans=max_scans, warnings_are_errors=warnings_are_errors)
    library = _library()
    handle = _Settings(given)
    samples = np.ascontiguousarray(picture, dtype=np.float64)
    if samples.ndim not in (2, 3):
        raise ValueError(f"a picture is (height, width) or (height, width, channels), not {samples.shape}")
    data = Path(source).read_bytes() if isinstance(source, (str, os.PathLike)) else bytes(source)  # type: ignore[arg-type]
    result = ctypes.c_void_p()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_project(data, len(data), handle.handle,
                                     samples.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), samples.shape[0],
                                     samples.shape[1], samples.shape[2] if samples.ndim > 2 else 1,
                                     ctypes.byref(result), message, _MESSAGE)
    _raise(status, message)
    try:
        return _decoded(library, result)
    finally:
        library.unround_result_free(result)


def to_rgb(planes: npt.ArrayLike) -> Array:
    """JFIF's RGB (H, W, 3) of Y, Cb and Cr planes (3, H, W) (docs/math.md 8)."""
    values = np.ascontiguousarray(planes, dtype=np.float64)
    if values.ndim != 3 or values.shape[0] != 3:
        raise ValueError(f"the planes are (3, height, width), not {values.shape}")
    out = np.empty((values.shape[1], values.shape[2], 3))
    p = ctypes.POINTER(ctypes.c_double)
    _library().unround_to_rgb(values.ctypes.data_as(p), values.shape[1], values.shape[2], out.ctypes.data_as(p))
    return out


def to_ycbcr(picture: npt.ArrayLike) -> Array:
    """JFIF's Y, Cb and Cr planes (3, H, W) of an RGB picture (H, W, 3)."""
    values = np.ascontiguousarray(picture, dtype=np.float64)
    if values.ndim != 3 or values.shape[2] != 3:
        raise ValueError(f"the picture is (height, width, 3), not {values.shape}")
    out = np.empty((3, values.shape[0], values.shape[1]))
    p = ctypes.POINTER(ctypes.c_double)
    _library().unround_to_ycbcr(values.ctypes.data_as(p), values.shape[0], values.shape[1], out.ctypes.data_as(p))
    return out


# The command line's --dither and --dither-channels (docs/cli.md), as the interface's dither.
_DITHERS = {("blue-noise", None): 1, ("blue-noise", "apart"): 1, ("blue-noise", "together"): 2, ("none", None): 0}


def _dither(dither: str, channels: str | None) -> int:
    """The interface's dither of the command line's --dither and --dither-channels."""
    found = _DITHERS.get((dither, channels))
    if found is None:
        message = f"the dither is blue-noise, with the channels apart or together, or none, not {dither}" + (
            "" if channels is None else f" with the channels {channels}"
        )
        raise ValueError(message)
    return found


def pnm_bytes(picture: npt.ArrayLike, *, sixteen: bool = False, dither: str = "blue-noise",
              dither_channels: str | None = None) -> bytes:
    """A PNM file of the picture's samples, (height, width) grey or (height, width, 3) RGB, of 8
    bits, or of 16 (257 levels to a unit): each sample by the ordered dither of the blue-noise
    matrix (dither "blue-noise", the channels "apart" -- the default -- or "together") or rounded
    to the nearest level, halves away from 0 ("none"), clamped (docs/math.md 10). The levels are
    made on the GPU (unround_pnm)."""
    made = _dither(dither, dither_channels)
    samples = np.ascontiguousarray(picture, dtype=np.float64)
    if samples.ndim not in (2, 3):
        raise ValueError(f"a picture is (height, width) or (height, width, channels), not {samples.shape}")
    height, width = int(samples.shape[0]), int(samples.shape[1])
    channels = 1 if samples.ndim == 2 else int(samples.shape[2])
    library = _library()
    pointer = ctypes.POINTER(ctypes.c_uint8)()
    size = ctypes.c_uint64()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_pnm(samples.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), height, width, channels,
                                 1 if sixteen else 0, made, ctypes.byref(pointer), ctypes.byref(size), message,
                                 _MESSAGE)
    _raise(status, message)
    try:
        return ctypes.string_at(pointer, int(size.value))
    finally:
        library.unround_bytes_free(pointer, size)


def png_bytes(picture: npt.ArrayLike, *, sixteen: bool = False, dither: str = "blue-noise",
              dither_channels: str | None = None, compression: int | None = None,
              icc_profile: bytes | None = None) -> bytes:
    """A PNG file of the picture's samples, (height, width) or (height, width, channels) with 1 to 4
    channels, of 8 bits or 16, the levels made on the GPU as pnm_bytes makes them (unround_png).
    compression is zlib's level, 0 to 9, or None for its default; the ICC profile is written where
    it goes with the picture, and otherwise left out with an UnroundWarning."""
    level = -1 if compression is None else compression
    if not -1 <= level <= 9:
        raise ValueError(f"zlib's level is 0 to 9, or None, not {compression}")
    made = _dither(dither, dither_channels)
    samples = np.ascontiguousarray(picture, dtype=np.float64)
    if samples.ndim not in (2, 3):
        raise ValueError(f"a picture is (height, width) or (height, width, channels), not {samples.shape}")
    height, width = int(samples.shape[0]), int(samples.shape[1])
    channels = 1 if samples.ndim == 2 else int(samples.shape[2])
    profile = b"" if icc_profile is None else bytes(icc_profile)
    profile_buffer = (ctypes.c_uint8 * max(len(profile), 1)).from_buffer_copy(profile or b"\0")
    library = _library()
    pointer = ctypes.POINTER(ctypes.c_uint8)()
    size = ctypes.c_uint64()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_png(samples.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), height, width, channels,
                                 1 if sixteen else 0, made, level,
                                 profile_buffer if icc_profile is not None else None, len(profile),
                                 ctypes.byref(pointer), ctypes.byref(size), message, _MESSAGE)
    _raise(status, message)
    try:
        if message.value:
            warnings.warn(message.value.decode("utf-8", "replace"), UnroundWarning, stacklevel=2)
        return ctypes.string_at(pointer, int(size.value))
    finally:
        library.unround_bytes_free(pointer, size)


def tiff_bytes(picture: npt.ArrayLike, *, ycbcr: bool = False, icc_profile: bytes | None = None) -> bytes:
    """A TIFF of the picture's samples in binary64, bit for bit (unround_tiff): (height, width) or
    (height, width, channels) with 1 to 4 channels, an alpha last. With ycbcr, the three samples of
    a pixel are JFIF's Y, Cb and Cr, and the file says so. The ICC profile is embedded where it goes
    with the picture (jpegio.check_icc); otherwise it is left out, with an UnroundWarning."""
    samples = np.ascontiguousarray(picture, dtype=np.float64)
    if samples.ndim not in (2, 3):
        raise ValueError(f"a picture is (height, width) or (height, width, channels), not {samples.shape}")
    height, width = int(samples.shape[0]), int(samples.shape[1])
    channels = 1 if samples.ndim == 2 else int(samples.shape[2])
    profile = None if icc_profile is None else bytes(icc_profile)
    buffer = (ctypes.c_uint8 * len(profile)).from_buffer_copy(profile) if profile else None
    library = _library()
    pointer = ctypes.POINTER(ctypes.c_uint8)()
    size = ctypes.c_uint64()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_tiff(samples.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), height, width, channels,
                                  1 if ycbcr else 0, buffer, 0 if profile is None else len(profile),
                                  ctypes.byref(pointer), ctypes.byref(size), message, _MESSAGE)
    _raise(status, message)
    try:
        if message.value:
            warnings.warn(message.value.decode("utf-8", "replace"), UnroundWarning, stacklevel=2)
        return ctypes.string_at(pointer, int(size.value))
    finally:
        library.unround_bytes_free(pointer, size)


def main(arguments: list[str] | None = None) -> int:
    """The reference's command line (unround_main): outside this build's path, its exit status is
    3 (unsupported)."""
    import sys

    given = [argument.encode("utf-8") for argument in (sys.argv[1:] if arguments is None else arguments)]
    array = (ctypes.c_char_p * max(len(given), 1))(*given)
    return int(_library().unround_main(len(given), array))


def oriented(picture: npt.ArrayLike, orientation: int) -> Array:
    """The picture, (height, width) or (height, width, channels), turned upright as EXIF's
    orientation says (unround_orient): 1 to 8, or 0 where the file has none, which is 1; from 5 on,
    the rows become columns. Every sample of the result is one of the picture's, bit for bit."""
    samples = np.ascontiguousarray(picture, dtype=np.float64)
    if samples.ndim not in (2, 3):
        raise ValueError(f"a picture is (height, width) or (height, width, channels), not {samples.shape}")
    if not -(2**31) <= orientation < 2**31:
        raise ValueError(f"an EXIF orientation is 1 to 8, or 0 for none, not {orientation}")
    height, width = int(samples.shape[0]), int(samples.shape[1])
    channels = 1 if samples.ndim == 2 else int(samples.shape[2])
    turned = np.empty(samples.size, dtype=np.float64)
    rows, columns = ctypes.c_uint64(), ctypes.c_uint64()
    message = ctypes.create_string_buffer(_MESSAGE)
    doubles = ctypes.POINTER(ctypes.c_double)
    library = _library()
    status = library.unround_orient(samples.ctypes.data_as(doubles), height, width, channels, orientation,
                                    turned.ctypes.data_as(doubles), ctypes.byref(rows), ctypes.byref(columns), message,
                                    _MESSAGE)
    _raise(status, message)
    shape = (int(rows.value), int(columns.value)) + (() if samples.ndim == 2 else (channels,))
    return turned.reshape(shape)


def solve_levels(image: jpegio.Image, settings: Settings | list[str] | None = None, *, sixteen: bool = False,
                 dither: str = "blue-noise", dither_channels: str | None = None) -> npt.NDArray:
    """The reconstruction as 8-bit (uint8) or 16-bit (uint16) levels, (height, width) grey or
    (height, width, channels), quantized on the GPU as pnm_bytes quantizes a picture: only the
    levels are copied back (include/unround_b200.h, unround_b200_solve_levels)."""
    library = _library()
    handle = _settings_of(settings)
    made = _dither(dither, dither_channels)
    given, kept = _input_of(image)
    sizes = (ctypes.c_uint64 * 3)()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_b200_solve_levels(ctypes.byref(given), handle.handle, int(sixteen), made, None, 0, sizes,
                                               message, _MESSAGE)
    _raise(status, message)
    height, width, channels = (int(v) for v in sizes)
    out = np.empty((height, width, channels), dtype=np.uint16 if sixteen else np.uint8)
    status = library.unround_b200_solve_levels(ctypes.byref(given), handle.handle, int(sixteen), made,
                                               out.ctypes.data_as(ctypes.c_void_p), out.nbytes, sizes, message,
                                               _MESSAGE)
    _raise(status, message)
    del kept
    if sixteen:
        out = out.byteswap()  # the interface's most significant byte first
    return out[:, :, 0] if channels == 1 else out


def solve_samples(levels: npt.ArrayLike, bits: int = 8, settings: Settings | list[str] | None = None) -> Decoded:
    """A picture of rounded samples -- a PNG file's levels, (height, width) grey or (height, width,
    channels) with 2 to 4 channels (an alpha last) -- reconstructed on the GPU within the
    intervals of its samples (include/unround_b200.h, unround_b200_solve_samples; docs/math.md
    11): TV or TGV as the settings say, with the defaults of PNG files."""
    values = np.ascontiguousarray(levels, dtype=np.uint16)
    if values.ndim == 2:
        values = values[:, :, np.newaxis]
    if values.ndim != 3:
        raise ValueError(f"levels are (height, width) or (height, width, channels), not {values.shape}")
    library = _library()
    handle = _settings_of(settings)
    result = ctypes.c_void_p()
    message = ctypes.create_string_buffer(_MESSAGE)
    rows, columns, channels = values.shape
    status = library.unround_b200_solve_samples(values.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), rows, columns,
                                                channels, int(bits), handle.handle, _OBSERVER(), None,
                                                ctypes.byref(result), message, _MESSAGE)
    _raise(status, message)
    try:
        return _decoded(library, result, problems=False)
    finally:
        library.unround_result_free(result)


def measure_samples(levels: npt.ArrayLike, bits: int = 8, settings: Settings | list[str] | None = None, *,
                    warmup: int = 3, iterations: int = 100) -> Timing:
    """The iteration loop of solve_samples alone on the GPU, timed by CUDA events
    (unround_b200_measure_samples): grey (height, width) or RGB (height, width, 3) levels."""
    values = np.ascontiguousarray(levels, dtype=np.uint16)
    if values.ndim == 2:
        values = values[:, :, np.newaxis]
    library = _library()
    handle = _settings_of(settings)
    timing = _Timing()
    message = ctypes.create_string_buffer(_MESSAGE)
    rows, columns, channels = values.shape
    status = library.unround_b200_measure_samples(values.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), rows,
                                                  columns, channels, int(bits), handle.handle, warmup, iterations,
                                                  ctypes.byref(timing), message, _MESSAGE)
    _raise(status, message)
    return Timing(timing.milliseconds, timing.dual_milliseconds, timing.primal_milliseconds, int(timing.iterations),
                  int(timing.launches_per_iteration), int(timing.samples), int(timing.pixels), int(timing.device_bytes))
