"""The JPEG reader (unround_jpeg_read, unround_jpeg_decode_planes; csrc/jpeg_reader.cpp) pinned
against libjpeg-turbo, which Pillow carries: files that Pillow writes (the reference's own test
cases, python/tests/test_jpegio.py:68-123: grey and colour 4:4:4, 4:2:2, 4:2:0, qualities 10, 50
and 90, sequential and progressive, 1x1 to 48x33), read here and decoded by libjpeg-turbo.

The reader's coefficients, dequantized and inverse-transformed exactly, must give libjpeg's
samples within 1 (its integer inverse DCT), sample for sample: Y and 4:4:4 chroma directly
(libjpeg's output in YCbCr), subsampled chroma through the triangle filter that libjpeg's fancy
upsampling applies, within 2. With every step of a custom table at 100, a coefficient one off
moves some sample of its block by at least 12, so those files pin every coefficient exactly.
The quantization tables must be Pillow's; the structure (sizes, blocks, sampling, colour space)
the reference test's. Restart intervals, EXIF orientation, a multi-marker ICC profile, the
limits, refusals and damaged files as the reference tests them. No GPU is needed."""

from __future__ import annotations

import io
import zlib
from typing import NamedTuple

import numpy as np
import pytest
from PIL import Image as PILImage

from unround import jpegio


def picture(seed: int, height: int, width: int, channels: int) -> np.ndarray:
    """Waves, steps and noise (as the reference's test pictures are made)."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:height, 0:width].astype(np.float64)
    layers = []
    for channel in range(channels):
        phase = rng.uniform(0.0, 2.0 * np.pi)
        value = 128.0 + 70.0 * np.sin(x / (9.0 + channel) + phase) * np.cos(y / 7.0)
        value += 60.0 * (((x // 13) + (y // 11)) % 3 == 0)
        value += rng.integers(-24, 25, size=(height, width))
        layers.append(np.clip(value, 0, 255))
    stacked = np.stack(layers, axis=-1).astype(np.uint8)
    return stacked[..., 0] if channels == 1 else stacked


def encode(pixels: np.ndarray, **options: object) -> bytes:
    buffer = io.BytesIO()
    PILImage.fromarray(pixels).save(buffer, format="JPEG", **options)
    return buffer.getvalue()


def libjpeg_planes(data: bytes) -> np.ndarray:
    """libjpeg-turbo's decoded samples: grey, or Y, Cb and Cr (no colour conversion)."""
    opened = PILImage.open(io.BytesIO(data))
    if opened.mode != "L":
        opened.draft("YCbCr", opened.size)
    return np.asarray(opened).astype(np.int64)


def upsampled(plane: np.ndarray, down: int, across: int, height: int, width: int) -> np.ndarray:
    """A subsampled plane brought to full size by the triangle filter (each output sample 3/4 of
    the nearer input and 1/4 of the further, per direction), in binary64."""
    out = plane.astype(np.float64)
    if across == 2:
        left = np.concatenate([out[:, :1], out[:, :-1]], axis=1)
        right = np.concatenate([out[:, 1:], out[:, -1:]], axis=1)
        wide = np.empty((out.shape[0], 2 * out.shape[1]))
        wide[:, 0::2] = 0.75 * out + 0.25 * left
        wide[:, 1::2] = 0.75 * out + 0.25 * right
        out = wide
    if down == 2:
        up = np.concatenate([out[:1], out[:-1]], axis=0)
        below = np.concatenate([out[1:], out[-1:]], axis=0)
        tall = np.empty((2 * out.shape[0], out.shape[1]))
        tall[0::2] = 0.75 * out + 0.25 * up
        tall[1::2] = 0.75 * out + 0.25 * below
        out = tall
    return out[:height, :width]


def exact_plane(component: jpegio.Component) -> np.ndarray:
    """The exact inverse DCT of a component's dequantized coefficients, + 128, unrounded."""
    n = np.arange(8)
    basis = np.cos((2 * n[:, None] + 1) * n[None, :] * np.pi / 16) * np.where(n == 0, np.sqrt(1 / 8), 0.5)[None, :]
    f = component.coefficients.astype(np.float64) * component.quant_table.astype(np.float64)
    blocks = np.einsum("yv,abvu,xu->abyx", basis, f, basis) + 128.0
    rows, columns = blocks.shape[:2]
    return blocks.transpose(0, 2, 1, 3).reshape(rows * 8, columns * 8)


def check_against_libjpeg(data: bytes, image: jpegio.Image, subsampled_tolerance: float = 2.0) -> None:
    theirs = libjpeg_planes(data)
    h, w = image.height, image.width
    if theirs.ndim == 2:
        theirs = theirs[..., None]
    for index, component in enumerate(image.components):
        ours = np.clip(np.rint(exact_plane(component)), 0, 255)
        down = image.max_v_samp_factor // component.v_samp_factor
        across = image.max_h_samp_factor // component.h_samp_factor
        if down == 1 and across == 1:
            assert np.abs(ours[:h, :w] - theirs[..., index]).max() <= 1
        else:
            near = upsampled(ours[: component.height, : component.width], down, across, h, w)
            assert np.abs(near - theirs[..., index]).max() <= subsampled_tolerance


class Case(NamedTuple):
    mode: str
    subsampling: int
    quality: int
    progressive: bool
    height: int
    width: int

    def __str__(self) -> str:
        coding = "progressive" if self.progressive else "sequential"
        return f"{self.mode}-{self.subsampling}-q{self.quality}-{coding}-{self.height}x{self.width}"


CASES = [
    Case(mode, subsampling, quality, progressive, height, width)
    for mode, subsampling in [("L", 0), ("RGB", 0), ("RGB", 1), ("RGB", 2)]
    for quality in (10, 50, 90)
    for progressive in (False, True)
    for height, width in [(1, 1), (8, 8), (21, 37), (48, 33)]
]


@pytest.mark.parametrize("case", CASES, ids=str)
def test_coefficients_match_libjpeg(case: Case) -> None:
    channels = 1 if case.mode == "L" else 3
    seed = zlib.crc32(str(case).encode())
    data = encode(picture(seed, case.height, case.width, channels), quality=case.quality,
                  subsampling=case.subsampling, progressive=case.progressive)
    ours = jpegio.read(data)
    assert (ours.width, ours.height) == (case.width, case.height)
    assert ours.progressive == case.progressive
    assert ours.color_space == (jpegio.ColorSpace.GRAYSCALE if channels == 1 else jpegio.ColorSpace.YCBCR)
    assert ours.warnings == 0 and ours.warning == ""
    assert len(ours.components) == channels
    tables = PILImage.open(io.BytesIO(data)).quantization
    for component in ours.components:
        assert component.coefficients.dtype == np.int16
        np.testing.assert_array_equal(component.quant_table.reshape(64), tables[component.quant_table_slot])
        assert component.height_in_blocks == -(-component.height // 8)
        assert component.width_in_blocks == -(-component.width // 8)
    if channels == 3:
        expected = {0: (1, 1), 1: (2, 1), 2: (2, 2)}[case.subsampling]
        assert (ours.components[0].h_samp_factor, ours.components[0].v_samp_factor) == expected
        assert all((c.h_samp_factor, c.v_samp_factor) == (1, 1) for c in ours.components[1:])
    check_against_libjpeg(data, ours)


@pytest.mark.parametrize("mode, subsampling", [("L", 0), ("RGB", 0), ("RGB", 2)])
@pytest.mark.parametrize("progressive", [False, True])
def test_every_coefficient_is_exact_with_coarse_steps(mode: str, subsampling: int, progressive: bool) -> None:
    # Steps of 100: a coefficient one off moves its block by at least 100 / 8 somewhere.
    pixels = picture(7, 40, 56, 1 if mode == "L" else 3)
    tables = [[100] * 64] * (1 if mode == "L" else 2)
    data = encode(pixels, qtables=tables, subsampling=subsampling, progressive=progressive)
    ours = jpegio.read(data)
    theirs = libjpeg_planes(data)
    theirs = theirs[..., None] if theirs.ndim == 2 else theirs
    nonzero = 0
    for index, component in enumerate(ours.components):
        nonzero += int(np.count_nonzero(component.coefficients))
        if component.h_samp_factor == ours.max_h_samp_factor and component.v_samp_factor == ours.max_v_samp_factor:
            exact = exact_plane(component)[: ours.height, : ours.width]
            inside = (exact > 1) & (exact < 254)  # clamping hides nothing here
            assert np.abs(np.rint(exact) - theirs[..., index])[inside].max() <= 1
    assert nonzero > 100


def test_planes_are_the_inverse_dct_of_the_coefficients() -> None:
    for subsampling in (0, 1, 2):
        data = encode(picture(subsampling, 45, 70, 3), quality=40, subsampling=subsampling)
        image = jpegio.read(data)
        planes = jpegio.decode_planes(data)
        assert planes.warning == ""
        assert len(planes.planes) == len(image.components)
        for component, plane in zip(image.components, planes.planes, strict=True):
            rows, columns = component.height_in_blocks, component.width_in_blocks
            assert plane.shape == (rows * 8, columns * 8) and plane.dtype == np.uint8
            expected = np.clip(np.rint(exact_plane(component)), 0, 255)
            assert np.abs(plane.astype(np.float64) - expected).max() <= 1


@pytest.mark.parametrize("option", [{"restart_marker_blocks": 3}, {"restart_marker_rows": 1}])
@pytest.mark.parametrize("progressive", [False, True])
def test_restart_intervals(option: dict, progressive: bool) -> None:
    data = encode(picture(11, 37, 61, 3), quality=60, subsampling=2, progressive=progressive, **option)
    assert b"\xff\xdd" in data
    image = jpegio.read(data)
    assert image.warnings == 0
    check_against_libjpeg(data, image)


def test_exif_orientation_and_icc_profile() -> None:
    exif = PILImage.Exif()
    exif[0x0112] = 6
    profile = bytes(np.random.default_rng(3).integers(0, 256, 150_000, dtype=np.uint8))  # three APP2 markers
    data = encode(picture(1, 16, 24, 3), exif=exif.tobytes(), icc_profile=profile)
    image = jpegio.read(data)
    assert image.exif_orientation == 6
    assert image.icc_profile == profile
    plain = jpegio.read(encode(picture(1, 16, 24, 3)))
    assert plain.exif_orientation == 0 and plain.icc_profile is None


def test_what_cannot_be_read_raises() -> None:
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(b"")
    assert raised.value.kind is jpegio.ErrorKind.DECODE
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(b"not a jpeg file at all")
    assert raised.value.kind is jpegio.ErrorKind.DECODE
    buffer = io.BytesIO()
    PILImage.new("CMYK", (16, 16), (10, 20, 30, 40)).save(buffer, format="JPEG")
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(buffer.getvalue())
    assert raised.value.kind is jpegio.ErrorKind.UNSUPPORTED


def test_a_cut_file_warns_or_fails() -> None:
    data = encode(picture(5, 64, 64, 3), quality=80)
    image = jpegio.read(data[: len(data) // 2])
    assert image.warnings >= 1
    assert image.warning == "Premature end of JPEG file"
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(data[: len(data) // 2], warnings_are_errors=True)
    assert raised.value.kind is jpegio.ErrorKind.DECODE


def test_limits() -> None:
    data = encode(picture(2, 40, 50, 3), progressive=True)
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(data, max_pixels=40 * 50 - 1)
    assert raised.value.kind is jpegio.ErrorKind.LIMIT
    assert jpegio.read(data, max_pixels=40 * 50).width == 50
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(data, max_scans=2)
    assert raised.value.kind is jpegio.ErrorKind.LIMIT
    with pytest.raises(jpegio.JpegioError) as raised:
        jpegio.read(data, max_pixels=-1)
    assert raised.value.kind is jpegio.ErrorKind.ARGUMENT


def test_arrays_are_read_only_copies() -> None:
    image = jpegio.read(encode(picture(4, 16, 16, 1)))
    component = image.components[0]
    assert not component.coefficients.flags.writeable and not component.quant_table.flags.writeable
    with pytest.raises(ValueError):
        component.coefficients[0, 0, 0, 0] = 1


def test_damaged_files_give_an_image_or_an_error() -> None:
    # Seeded damage: bytes changed, cut or dropped; every read ends with an image or JpegioError.
    rng = np.random.default_rng(17)
    originals = [encode(picture(s, 24, 40, 3), quality=70, progressive=bool(s % 2)) for s in range(4)]
    for trial in range(300):
        data = bytearray(originals[trial % len(originals)])
        for _ in range(int(rng.integers(1, 6))):
            at = int(rng.integers(0, len(data)))
            data[at] = int(rng.integers(0, 256))
        if trial % 3 == 0:
            data = data[: int(rng.integers(2, len(data)))]
        try:
            image = jpegio.read(bytes(data))
        except jpegio.JpegioError:
            continue
        for component in image.components:
            assert component.coefficients.shape[2:] == (8, 8)
