"""Files reconstructed through unround_decode on the GPU: a JPEG file (Pillow-written, so
libjpeg-turbo's encoder) against the reference's own solver (oracle/_ref) on the coefficients of
the same file, with the bar of the array path (relative L2 <= 1e-4, max |difference| <= 2e-3, the
same iterations, every coefficient within its interval); the file's metadata (EXIF orientation,
ICC profile) on the result. A PNG file against the reference's solver of rounded samples on the
levels the file holds. And png_bytes: the PNG file of a picture holds the PNM file's samples
(python/tests/test_native.py:683-700 of the reference)."""

import io
import warnings

import numpy as np
import pytest
from PIL import Image as PILImage

from oracle import reference

pytestmark = pytest.mark.gpu


def _picture(seed: int, height: int, width: int, channels: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:height, 0:width].astype(np.float64)
    layers = [np.clip(120 + 60 * np.sin(x / (7 + c) + rng.uniform(0, 6)) * np.cos(y / 9) + 40 * ((x // 11 + y // 13) % 2)
                      + rng.normal(0, 3, (height, width)), 0, 255) for c in range(channels)]
    stacked = np.rint(np.stack(layers, -1)).astype(np.uint8)
    return stacked[..., 0] if channels == 1 else stacked


def _jpeg(pixels: np.ndarray, **options: object) -> bytes:
    buffer = io.BytesIO()
    PILImage.fromarray(pixels).save(buffer, format="JPEG", **options)
    return buffer.getvalue()


@pytest.mark.parametrize("channels, subsampling, progressive, options", [
    (1, 0, False, ["--method", "tv", "--iterations", "80", "--tolerance", "0"]),
    (3, 2, True, ["--method", "tgv", "--iterations", "60", "--tolerance", "0"]),
    (3, 1, False, ["--method", "tgv", "--iterations", "40", "--tolerance", "0", "--channels", "apart"]),
])
def test_a_jpeg_file_against_the_reference_solver(channels, subsampling, progressive, options):
    from unround import jpegio, native

    data = _jpeg(_picture(channels + subsampling, 53, 77, channels), quality=60, subsampling=subsampling,
                 progressive=progressive)
    ours = native.decode(data, options)
    image = jpegio.read(data)
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor)
                  for c in image.components]
    theirs = reference.solve(image.height, image.width, int(image.color_space), components, options)
    difference = ours.canvas - theirs.canvas
    assert np.linalg.norm(difference) / np.linalg.norm(theirs.canvas) <= 1e-4
    assert np.max(np.abs(difference)) <= 2e-3
    assert ours.result.iterations == theirs.iterations
    for index, problem in enumerate(ours.problems):
        c = ours.coefficients[index]
        assert np.all(c >= problem.lower) and np.all(c <= problem.upper)
    # The file path and the array path are one solve.
    again = native.solve(image, options)
    np.testing.assert_array_equal(again.canvas, ours.canvas)
    assert ours.input_format == "jpeg"


def test_a_jpeg_file_s_metadata_on_the_result():
    from unround import native

    exif = PILImage.Exif()
    exif[0x0112] = 8
    profile = bytes(range(256)) * 3
    data = _jpeg(_picture(1, 24, 40, 3), exif=exif.tobytes(), icc_profile=profile)
    decoded = native.decode(data, ["--method", "tv", "--iterations", "10"])
    assert decoded.exif_orientation == 8
    assert decoded.icc_profile == profile
    upright = native.oriented(decoded.picture, decoded.exif_orientation)
    np.testing.assert_array_equal(upright, np.rot90(decoded.picture, 1))


def test_a_cut_jpeg_file_warns():
    from unround import native

    data = _jpeg(_picture(2, 64, 64, 1), quality=80)
    with warnings.catch_warnings(record=True) as seen:
        warnings.simplefilter("always")
        native.decode(data[: len(data) * 2 // 3], ["--method", "tv", "--iterations", "5"])
    assert any("Premature end of JPEG file" in str(w.message) for w in seen)
    with pytest.raises(native.UnroundError) as raised:
        native.decode(data[: len(data) * 2 // 3], ["--method", "tv", "--iterations", "5"], warnings_are_errors=True)
    assert raised.value.status == native.Status.READ


@pytest.mark.parametrize("mode", ["L", "LA", "RGB", "RGBA", "I;16"])
def test_a_png_file_against_the_reference_solver(mode):
    from unround import native

    channels = {"L": 1, "LA": 2, "RGB": 3, "RGBA": 4, "I;16": 1}[mode]
    pixels = _picture(5, 36, 44, channels)
    bits = 8
    if mode == "I;16":  # 16 bits: the 8-bit picture spread over the levels, with a little noise
        bits = 16
        noise = np.random.default_rng(6).integers(0, 200, size=pixels.shape)
        pixels = (pixels.astype(np.int64) * 257 + noise).clip(0, 65535).astype(np.uint16)
    buffer = io.BytesIO()
    PILImage.fromarray(pixels).save(buffer, format="PNG")
    assert PILImage.open(io.BytesIO(buffer.getvalue())).mode == mode
    options = ["--method", "tgv", "--iterations", "120", "--tolerance", "0"]
    ours = native.decode(buffer.getvalue(), options)
    assert ours.input_format == "png" and ours.bits == bits
    theirs = reference.solve_samples(pixels, bits, options)
    got = ours.canvas.reshape(theirs.canvas.shape)
    assert np.linalg.norm(got - theirs.canvas) / np.linalg.norm(theirs.canvas) <= 1e-4
    assert np.max(np.abs(got - theirs.canvas)) <= 2e-3
    np.testing.assert_array_equal(native.solve_samples(pixels, bits, options).canvas, ours.canvas)


@pytest.mark.parametrize("sixteen", [False, True])
@pytest.mark.parametrize("channels", [1, 3])
def test_the_png_holds_the_pnm_s_samples(sixteen, channels):
    from unround import native

    rng = np.random.default_rng(channels + 2 * sixteen)
    shape = (13, 17) if channels == 1 else (13, 17, 3)
    picture = rng.uniform(-10, 265, size=shape)
    for dither in ("none", "blue-noise"):
        png = native.png_bytes(picture, sixteen=sixteen, dither=dither)
        pnm = native.pnm_bytes(picture, sixteen=sixteen, dither=dither)
        body = pnm.split(b"\n", 3)[3]
        expected = np.frombuffer(body, dtype=">u2" if sixteen else np.uint8).astype(np.int64).reshape(shape)
        opened = PILImage.open(io.BytesIO(png))
        if sixteen and channels == 3:
            continue  # Pillow holds 16-bit samples of grey alone; the reader tests cover these files
        np.testing.assert_array_equal(np.asarray(opened).astype(np.int64), expected)
    with pytest.raises(ValueError):
        native.png_bytes(picture, compression=10)
