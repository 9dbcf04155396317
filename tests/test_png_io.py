"""PNG reading and writing (unround_jpegio_read_png, unround_jpegio_write_png; csrc/png_io.cpp)
pinned against Pillow's PNG codec: files Pillow writes read back as Pillow reads them; files
written here read back by Pillow as the levels given; interlaced (Adam7) and 1-, 2- and 4-bit
files from a small encoder of the test, checked by Pillow first. A palette file is refused as the
reference refuses it (c/jpegio/src/png.c:428-444), a tRNS chunk is warned about, broken files fail,
and the ICC profile of an iCCP chunk comes back, or is left out of a file where it does not go with
the picture. No GPU is needed."""

from __future__ import annotations

import ctypes
import io
import struct
import zlib

import numpy as np
import pytest
from PIL import Image as PILImage

from unround import native


class _PngImage(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("channels", ctypes.c_int32),
        ("bits", ctypes.c_int32),
        ("samples", ctypes.POINTER(ctypes.c_uint16)),
        ("icc_profile", ctypes.POINTER(ctypes.c_uint8)),
        ("icc_profile_size", ctypes.c_uint64),
    ]


class _Png(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("channels", ctypes.c_int32),
        ("bits", ctypes.c_int32),
        ("compression", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("samples", ctypes.c_void_p),
        ("icc_profile", ctypes.POINTER(ctypes.c_uint8)),
        ("icc_profile_size", ctypes.c_uint64),
    ]


class _Bytes(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(ctypes.c_uint8)), ("size", ctypes.c_uint64)]


def _library() -> ctypes.CDLL:
    library = native._library()
    library.unround_jpegio_read_png.restype = ctypes.c_int32
    library.unround_jpegio_read_png.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint64,
                                                ctypes.POINTER(_PngImage), ctypes.c_char_p, ctypes.c_size_t]
    library.unround_jpegio_png_image_free.argtypes = [ctypes.POINTER(_PngImage)]
    library.unround_jpegio_write_png.restype = ctypes.c_int32
    library.unround_jpegio_write_png.argtypes = [ctypes.POINTER(_Png), ctypes.POINTER(_Bytes), ctypes.c_char_p,
                                                 ctypes.c_size_t]
    library.unround_jpegio_bytes_free.argtypes = [ctypes.POINTER(_Bytes)]
    return library


def read_png(data: bytes, max_pixels: int = 0) -> tuple[int, np.ndarray | None, int, bytes | None, str]:
    """status, levels (height, width, channels), bits, ICC profile, message."""
    library = _library()
    image = _PngImage()
    message = ctypes.create_string_buffer(512)
    status = library.unround_jpegio_read_png(data, len(data), max_pixels, ctypes.byref(image), message, 512)
    text = message.value.decode()
    if status != 0:
        return status, None, 0, None, text
    try:
        count = image.height * image.width * image.channels
        levels = np.ctypeslib.as_array(image.samples, shape=(count,)).copy().reshape(image.height, image.width,
                                                                                      image.channels)
        icc = ctypes.string_at(image.icc_profile, image.icc_profile_size) if image.icc_profile_size else None
        return status, levels, int(image.bits), icc, text
    finally:
        library.unround_jpegio_png_image_free(ctypes.byref(image))


def write_png(levels: np.ndarray, bits: int, compression: int = -1, icc: bytes | None = None) -> tuple[int, bytes, str]:
    library = _library()
    samples = np.ascontiguousarray(levels, dtype=np.uint8 if bits == 8 else np.uint16)
    height, width = samples.shape[:2]
    channels = 1 if samples.ndim == 2 else samples.shape[2]
    profile = (ctypes.c_uint8 * len(icc)).from_buffer_copy(icc) if icc else None
    png = _Png(width, height, channels, bits, compression, 0, samples.ctypes.data, profile,
               len(icc) if icc else 0)
    out = _Bytes()
    message = ctypes.create_string_buffer(512)
    status = library.unround_jpegio_write_png(ctypes.byref(png), ctypes.byref(out), message, 512)
    try:
        return status, ctypes.string_at(out.data, out.size) if status == 0 else b"", message.value.decode()
    finally:
        library.unround_jpegio_bytes_free(ctypes.byref(out))


def pillow_png(array: np.ndarray, **options: object) -> bytes:
    buffer = io.BytesIO()
    PILImage.fromarray(array).save(buffer, format="PNG", **options)
    return buffer.getvalue()


def chunk(kind: bytes, body: bytes) -> bytes:
    return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)


def encoded(levels: np.ndarray, bits: int, *, interlaced: bool = False, colour_type: int | None = None,
            extra: bytes = b"") -> bytes:
    """A PNG file of the levels (height, width, channels) from the specification, rows unfiltered."""
    height, width, channels = levels.shape
    kind = colour_type if colour_type is not None else {1: 0, 2: 4, 3: 2, 4: 6}[channels]

    def rows(part: np.ndarray) -> bytes:
        out = b""
        for row in part:
            flat = row.reshape(-1)
            if bits == 16:
                line = b"".join(int(v).to_bytes(2, "big") for v in flat)
            elif bits == 8:
                line = bytes(int(v) for v in flat)
            else:
                text = "".join(format(int(v), f"0{bits}b") for v in flat)
                text += "0" * (-len(text) % 8)
                line = int(text, 2).to_bytes(len(text) // 8, "big")
            out += b"\0" + line
        return out

    if interlaced:
        passes = [(0, 0, 8, 8), (0, 4, 8, 8), (4, 0, 8, 4), (0, 2, 4, 4), (2, 0, 4, 2), (0, 1, 2, 2), (1, 0, 2, 1)]
        raw = b"".join(rows(levels[r0::dr, c0::dc]) for r0, c0, dr, dc in passes if levels[r0::dr, c0::dc].size)
    else:
        raw = rows(levels)
    header = struct.pack(">IIBBBBB", width, height, bits, kind, 0, 0, 1 if interlaced else 0)
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", header) + extra + chunk(b"IDAT", zlib.compress(raw))
            + chunk(b"IEND", b""))


def profile(space: bytes = b"RGB ") -> bytes:
    """A minimal ICC profile of version 4 with no tags: what a reader checks, and nothing more."""
    header = bytearray(132)
    struct.pack_into(">I", header, 0, 132)
    header[8] = 4
    header[12:16] = b"mntr"
    header[16:20] = space
    header[20:24] = b"XYZ "
    header[36:40] = b"acsp"
    return bytes(header)


@pytest.mark.parametrize("mode, shape, dtype", [
    ("L", (23, 31), np.uint8), ("LA", (23, 31, 2), np.uint8), ("RGB", (19, 40, 3), np.uint8),
    ("RGBA", (17, 9, 4), np.uint8), ("I;16", (21, 33), np.uint16),
])
@pytest.mark.parametrize("optimize", [False, True])
def test_files_pillow_writes(mode: str, shape: tuple[int, ...], dtype: type, optimize: bool) -> None:
    rng = np.random.default_rng(len(mode) * 7 + int(optimize))
    top = 65535 if dtype is np.uint16 else 255
    array = rng.integers(0, top + 1, size=shape).astype(dtype)
    data = pillow_png(array, optimize=optimize)
    assert PILImage.open(io.BytesIO(data)).mode == mode
    status, levels, bits, icc, message = read_png(data)
    assert status == 0 and message == "" and icc is None
    assert bits == (16 if dtype is np.uint16 else 8)
    np.testing.assert_array_equal(levels.reshape(array.shape), array)


@pytest.mark.parametrize("bits", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("interlaced", [False, True])
def test_grey_of_every_depth_interlaced_or_not(bits: int, interlaced: bool) -> None:
    levels = np.random.default_rng(bits).integers(0, 2**bits, size=(13, 19, 1))
    data = encoded(levels, bits, interlaced=interlaced)
    theirs = np.asarray(PILImage.open(io.BytesIO(data))).astype(np.int64)
    scale = {1: 1, 2: 85, 4: 17, 8: 1, 16: 1}[bits]
    np.testing.assert_array_equal(theirs, levels[..., 0] * scale)  # the test's encoder, as Pillow reads it
    status, ours, read_bits, _, _ = read_png(data)
    assert status == 0 and read_bits == bits
    np.testing.assert_array_equal(ours, levels)


@pytest.mark.parametrize("channels, bits", [(3, 16), (4, 16), (2, 16), (3, 8), (4, 8)])
def test_colour_interlaced(channels: int, bits: int) -> None:
    levels = np.random.default_rng(channels * bits).integers(0, 2**bits, size=(11, 14, channels))
    status, ours, read_bits, _, _ = read_png(encoded(levels, bits, interlaced=True))
    assert status == 0 and read_bits == bits
    np.testing.assert_array_equal(ours, levels)


@pytest.mark.parametrize("channels", [1, 2, 3, 4])
@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("compression", [-1, 0, 9])
def test_files_written_here_read_back(channels: int, bits: int, compression: int) -> None:
    rng = np.random.default_rng(channels + bits + compression)
    y, x = np.mgrid[0:29, 0:37]
    smooth = (x * 3 + y * 5)[..., None] + np.arange(channels) * 11  # rows that the filters predict
    levels = (smooth + rng.integers(0, 3, size=(29, 37, channels))) % (2**bits)
    status, data, message = write_png(levels, bits, compression)
    assert status == 0 and message == ""
    status, ours, read_bits, _, _ = read_png(data)
    assert status == 0 and read_bits == bits
    np.testing.assert_array_equal(ours, levels)
    opened = PILImage.open(io.BytesIO(data))
    if bits == 8 or channels == 1:  # Pillow holds 16-bit samples of grey alone
        theirs = np.asarray(opened).astype(np.int64).reshape(29, 37, channels)
        np.testing.assert_array_equal(theirs, levels)


def test_icc_profiles() -> None:
    levels = np.random.default_rng(1).integers(0, 256, size=(8, 9, 3))
    given = profile()
    status, data, message = write_png(levels, 8, icc=given)
    assert status == 0 and message == ""
    assert PILImage.open(io.BytesIO(data)).info["icc_profile"] == given
    assert read_png(data)[3] == given
    # A grey profile does not go with RGB: the file is written without it, and the message says why.
    status, data, message = write_png(levels, 8, icc=profile(b"GRAY"))
    assert status == 0 and "not written" in message
    assert "icc_profile" not in PILImage.open(io.BytesIO(data)).info
    assert read_png(data)[3] is None


def test_refusals_and_warnings() -> None:
    palette = PILImage.fromarray(np.zeros((4, 4), np.uint8)).convert("P")
    buffer = io.BytesIO()
    palette.save(buffer, format="PNG")
    status, _, _, _, message = read_png(buffer.getvalue())
    assert status == 3 and "palette" in message
    levels = np.random.default_rng(2).integers(0, 256, size=(5, 6, 3))
    with_trns = encoded(levels, 8, extra=chunk(b"tRNS", b"\0\1\0\2\0\3"))
    status, ours, _, _, message = read_png(with_trns)
    assert status == 0 and message == "the transparent colour of the tRNS chunk is not taken"
    np.testing.assert_array_equal(ours, levels)
    plain = encoded(levels, 8)
    assert read_png(plain, max_pixels=29)[0] == 4
    assert read_png(plain, max_pixels=30)[0] == 0
    broken = bytearray(plain)
    broken[20] ^= 0xFF  # inside IHDR: its CRC fails
    assert read_png(bytes(broken))[0] == 7
    assert read_png(plain[: len(plain) // 2])[0] == 7
    assert read_png(b"\x89PNG\r\n\x1a\n")[0] == 7
