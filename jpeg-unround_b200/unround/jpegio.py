"""A JPEG file's quantized components, as the reference package's unround.jpegio gives them.

The reference reads them with its C layer over libjpeg-turbo (python/src/unround/jpegio.py of
JPEG-Unround). This build carries no libjpeg-turbo: the entropy decoding that produces the
levels stays on the host, outside the GPU path, and `read` refuses with JpegioError. The data
classes are the same, so that a caller that has levels and tables (from libjpeg-turbo
elsewhere, or made in memory) builds an Image and passes it to unround.native.solve.
"""

from __future__ import annotations

import enum
from dataclasses import dataclass
from typing import Final

import numpy as np
import numpy.typing as npt

__all__ = ["ABI_VERSION", "ColorSpace", "Component", "ErrorKind", "Image", "JpegioError", "Planes", "decode_planes", "read"]

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


def read(data: bytes | bytearray | memoryview, **_: object) -> Image:
    """Refuses: reading a JPEG file needs libjpeg-turbo, which this build does not carry."""
    raise JpegioError(ErrorKind.UNSUPPORTED, "reading a JPEG file needs libjpeg-turbo, which this build does not carry")


def decode_planes(data: bytes | bytearray | memoryview, **_: object) -> Planes:
    """Refuses, as read() does."""
    raise JpegioError(ErrorKind.UNSUPPORTED, "decoding a JPEG file needs libjpeg-turbo, which this build does not carry")
