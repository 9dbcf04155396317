"""A JPEG file's quantized components, as the reference package's unround.jpegio gives them.

The reference reads them with its C layer over libjpeg-turbo (python/src/unround/jpegio.py of
JPEG-Unround). This build reads them with its own reader in the same library as the solver
(unround_jpeg_read, unround_jpeg_decode_planes; a Huffman decoder of baseline, extended and
progressive files written from ITU-T T.81): the same structures, statuses and data classes, so
that read() and decode_planes() are drop-ins. image_of builds an Image of levels made in memory.
"""

from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from typing import Final

import numpy as np
import numpy.typing as npt

__all__ = ["ABI_VERSION", "ColorSpace", "Component", "ErrorKind", "Image", "JpegioError", "LibraryNotFoundError",
           "Planes", "abi_version", "check_icc", "decode_planes", "libjpeg_version", "libpng_version", "read"]

ABI_VERSION: Final = 3


class ErrorKind(enum.IntEnum):
    """What went wrong, as unround_jpegio_status says it."""

    ARGUMENT = 1
    DECODE = 2
    UNSUPPORTED = 3
    LIMIT = 4
    MEMORY = 5
    ENCODE = 6


class ColorSpace(enum.IntEnum):
    """The color space of the components."""

    GRAYSCALE = 1
    YCBCR = 2
    RGB = 3


class JpegioError(Exception):
    """A JPEG file that could not be read."""

    def __init__(self, kind: ErrorKind, message: str) -> None:
        super().__init__(f"{message} ({kind.name.lower()})")
        self.kind = kind
        self.message = message


class LibraryNotFoundError(RuntimeError):
    """The shared library is not where this package looks for it."""


@dataclass(frozen=True, slots=True, eq=False)
class Component:
    """One component: its sampling factors, size, quantization table (8, 8) in natural order,
    and its levels (height_in_blocks, width_in_blocks, 8, 8), element [by, bx, v, u]."""

    id: int
    h_samp_factor: int
    v_samp_factor: int
    quant_table_slot: int
    width: int
    height: int
    quant_table: npt.NDArray[np.uint16]
    coefficients: npt.NDArray[np.int16]

    @property
    def width_in_blocks(self) -> int:
        return int(self.coefficients.shape[1])

    @property
    def height_in_blocks(self) -> int:
        return int(self.coefficients.shape[0])


@dataclass(frozen=True, slots=True, eq=False)
class Image:
    """What read() returns: the picture's size, color space, sampling and components."""

    width: int
    height: int
    color_space: ColorSpace
    max_h_samp_factor: int
    max_v_samp_factor: int
    progressive: bool
    arithmetic: bool
    exif_orientation: int
    warnings: int
    warning: str
    components: tuple[Component, ...]
    icc_profile: bytes | None


@dataclass(frozen=True, slots=True, eq=False)
class Planes:
    """What decode_planes() returns: one array of 8-bit samples per component."""

    planes: tuple[npt.NDArray[np.uint8], ...]
    warning: str


def image_of(
    height: int,
    width: int,
    color_space: ColorSpace | int,
    components: list[tuple[npt.ArrayLike, npt.ArrayLike, int, int]],
) -> Image:
    """An Image of levels made in memory: components are (levels (rows, columns, 8, 8) int16,
    table (64,) or (8, 8) in natural order, h, v)."""
    made = []
    h_max = max(h for _, _, h, _ in components)
    v_max = max(v for _, _, _, v in components)
    for index, (levels, table, h, v) in enumerate(components):
        levels = np.ascontiguousarray(levels, dtype=np.int16)
        made.append(
            Component(
                id=index + 1,
                h_samp_factor=int(h),
                v_samp_factor=int(v),
                quant_table_slot=min(index, 1),
                width=-(-width * h // h_max),
                height=-(-height * v // v_max),
                quant_table=np.asarray(table, dtype=np.uint16).reshape(8, 8),
                coefficients=levels,
            )
        )
    return Image(
        width=width,
        height=height,
        color_space=ColorSpace(int(color_space)),
        max_h_samp_factor=h_max,
        max_v_samp_factor=v_max,
        progressive=False,
        arithmetic=False,
        exif_orientation=0,
        warnings=0,
        warning="",
        components=tuple(made),
        icc_profile=None,
    )


class _Options(ctypes.Structure):
    _fields_ = [("max_pixels", ctypes.c_uint64), ("max_scans", ctypes.c_int32), ("warnings_are_errors", ctypes.c_int32)]


class _Component(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_int32),
        ("h_samp_factor", ctypes.c_int32),
        ("v_samp_factor", ctypes.c_int32),
        ("quant_table_slot", ctypes.c_int32),
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("width_in_blocks", ctypes.c_uint32),
        ("height_in_blocks", ctypes.c_uint32),
        ("quant_table", ctypes.c_uint16 * 64),
        ("coefficients", ctypes.POINTER(ctypes.c_int16)),
    ]


class _Image(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("color_space", ctypes.c_int32),
        ("num_components", ctypes.c_int32),
        ("max_h_samp_factor", ctypes.c_int32),
        ("max_v_samp_factor", ctypes.c_int32),
        ("progressive", ctypes.c_int32),
        ("arithmetic", ctypes.c_int32),
        ("exif_orientation", ctypes.c_int32),
        ("warnings", ctypes.c_int32),
        ("components", _Component * 4),
        ("icc_profile", ctypes.POINTER(ctypes.c_uint8)),
        ("icc_profile_size", ctypes.c_uint64),
    ]


class _Plane(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("stride", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("samples", ctypes.POINTER(ctypes.c_uint8)),
    ]


class _Planes(ctypes.Structure):
    _fields_ = [("num_components", ctypes.c_int32), ("reserved", ctypes.c_int32), ("planes", _Plane * 4)]


_MESSAGE: Final = 512
_UINT64_MAX: Final = 2**64 - 1
_INT32_MAX: Final = 2**31 - 1


def _c_library() -> ctypes.CDLL:
    from unround import native  # the library is loaded (and its functions bound) there

    library = native._library()
    library.unround_jpeg_read.restype = ctypes.c_int32
    library.unround_jpeg_read.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_Options),
                                          ctypes.POINTER(_Image), ctypes.c_char_p, ctypes.c_size_t]
    library.unround_jpeg_image_free.restype = None
    library.unround_jpeg_image_free.argtypes = [ctypes.POINTER(_Image)]
    library.unround_jpeg_decode_planes.restype = ctypes.c_int32
    library.unround_jpeg_decode_planes.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_Options),
                                                   ctypes.POINTER(_Planes), ctypes.c_char_p, ctypes.c_size_t]
    library.unround_jpeg_planes_free.restype = None
    library.unround_jpeg_planes_free.argtypes = [ctypes.POINTER(_Planes)]
    library.unround_jpeg_abi_version.restype = ctypes.c_int32
    library.unround_jpeg_abi_version.argtypes = []
    library.unround_jpeg_libjpeg_version.restype = ctypes.c_char_p
    library.unround_jpeg_libjpeg_version.argtypes = []
    library.unround_jpeg_libpng_version.restype = ctypes.c_char_p
    library.unround_jpeg_libpng_version.argtypes = []
    library.unround_jpeg_check_icc.restype = ctypes.c_int32
    library.unround_jpeg_check_icc.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_char_p,
                                               ctypes.c_size_t]
    return library


def abi_version() -> int:
    """UNROUND_JPEGIO_ABI_VERSION of the library that is loaded."""
    return int(_c_library().unround_jpeg_abi_version())


def libjpeg_version() -> str:
    """What reads JPEG files in the library: this build's own reader (no libjpeg is carried)."""
    return _c_library().unround_jpeg_libjpeg_version().decode("ascii")


def libpng_version() -> str:
    """What reads and writes PNG files in the library: this build's own, and the zlib it uses."""
    return _c_library().unround_jpeg_libpng_version().decode("ascii")


def check_icc(profile: bytes, channels: int) -> str | None:
    """Why an ICC profile does not go with a picture of that many channels (1 or 2 grey, 3 or 4
    RGB), or None: the checks a reader makes of the profile of an iCCP chunk before it takes it;
    the PNG writer leaves out a profile that fails them."""
    if not 0 <= channels <= _INT32_MAX:
        raise ValueError(f"channels is {channels}, not 0 to 2**31 - 1")
    reason = ctypes.create_string_buffer(_MESSAGE)
    data = bytes(profile)
    accepted = _c_library().unround_jpeg_check_icc(data, len(data), channels, reason, _MESSAGE)
    return None if accepted == 1 else reason.value.decode("utf-8", "replace")


def _options(max_pixels: int, max_scans: int, *, warnings_are_errors: bool) -> _Options:
    if not 0 <= max_pixels <= _UINT64_MAX:
        raise JpegioError(ErrorKind.ARGUMENT, f"max_pixels is {max_pixels}, not 0 to 2**64 - 1")
    if not 0 <= max_scans <= _INT32_MAX:
        raise JpegioError(ErrorKind.ARGUMENT, f"max_scans is {max_scans}, not 0 to 2**31 - 1")
    return _Options(max_pixels, max_scans, 1 if warnings_are_errors else 0)


def _raise_for(status: int, message: str) -> None:
    if status != 0:
        try:
            kind = ErrorKind(status)
        except ValueError:
            kind = ErrorKind.DECODE
        raise JpegioError(kind, message)


def _read_only[T: np.generic](array: npt.NDArray[T]) -> npt.NDArray[T]:
    array.flags.writeable = False
    return array


def read(
    data: bytes | bytearray | memoryview,
    *,
    max_pixels: int = 0,
    max_scans: int = 0,
    warnings_are_errors: bool = False,
) -> Image:
    """The coefficients and metadata of a JPEG file in memory (unround_jpeg_read).

    max_pixels and max_scans limit what the file may declare (0 means the C layer's defaults,
    1 << 28 pixels and 500 scans), and warnings_are_errors makes corrupt data that the reader
    works around fail the read. The arrays are copies, read-only."""
    options = _options(max_pixels, max_scans, warnings_are_errors=warnings_are_errors)
    payload = bytes(data)
    library = _c_library()
    raw = _Image()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_jpeg_read(payload, len(payload), ctypes.byref(options), ctypes.byref(raw), message,
                                       _MESSAGE)
    text = message.value.decode("utf-8", "replace")
    _raise_for(status, text)
    try:
        components = []
        for index in range(raw.num_components):
            c = raw.components[index]
            count = c.height_in_blocks * c.width_in_blocks * 64
            levels = np.ctypeslib.as_array(c.coefficients, shape=(count,)).copy() if count else np.zeros(0, np.int16)
            components.append(
                Component(
                    id=int(c.id),
                    h_samp_factor=int(c.h_samp_factor),
                    v_samp_factor=int(c.v_samp_factor),
                    quant_table_slot=int(c.quant_table_slot),
                    width=int(c.width),
                    height=int(c.height),
                    quant_table=_read_only(np.array(c.quant_table, dtype=np.uint16).reshape(8, 8)),
                    coefficients=_read_only(levels.reshape(c.height_in_blocks, c.width_in_blocks, 8, 8)),
                )
            )
        icc = bytes(ctypes.string_at(raw.icc_profile, raw.icc_profile_size)) if raw.icc_profile_size else None
        return Image(
            width=int(raw.width),
            height=int(raw.height),
            color_space=ColorSpace(raw.color_space),
            max_h_samp_factor=int(raw.max_h_samp_factor),
            max_v_samp_factor=int(raw.max_v_samp_factor),
            progressive=bool(raw.progressive),
            arithmetic=bool(raw.arithmetic),
            exif_orientation=int(raw.exif_orientation),
            warnings=int(raw.warnings),
            warning=text,
            components=tuple(components),
            icc_profile=icc,
        )
    finally:
        library.unround_jpeg_image_free(ctypes.byref(raw))


def decode_planes(
    data: bytes | bytearray | memoryview,
    *,
    max_pixels: int = 0,
    max_scans: int = 0,
    warnings_are_errors: bool = False,
) -> Planes:
    """Each component's 8-bit samples (unround_jpeg_decode_planes): the inverse DCT of its
    dequantized coefficients, level-shifted and clamped, padded to whole blocks."""
    options = _options(max_pixels, max_scans, warnings_are_errors=warnings_are_errors)
    payload = bytes(data)
    library = _c_library()
    raw = _Planes()
    message = ctypes.create_string_buffer(_MESSAGE)
    status = library.unround_jpeg_decode_planes(payload, len(payload), ctypes.byref(options), ctypes.byref(raw),
                                                message, _MESSAGE)
    text = message.value.decode("utf-8", "replace")
    _raise_for(status, text)
    try:
        planes = []
        for index in range(raw.num_components):
            p = raw.planes[index]
            flat = np.ctypeslib.as_array(p.samples, shape=(p.height * p.stride,)).copy()
            planes.append(_read_only(flat.reshape(p.height, p.stride)[:, : p.width].copy()))
        return Planes(tuple(planes), text)
    finally:
        library.unround_jpeg_planes_free(ctypes.byref(raw))
