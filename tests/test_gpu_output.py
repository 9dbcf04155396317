"""8- and 16-bit output made on the GPU (unround_pnm through unround.native.pnm_bytes) against the
oracle (oracle/output.py, exact rationals), level for level, on the cases of the reference's own
tests (python/tests/test_native.py:569-640 of JPEG-Unround): halves away from 0, the 16-bit
products that round onto a half from below, the dither of the blue-noise matrix with the
channels apart and together, the files' headers, and the refusals."""

import math
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

from oracle import output

pytestmark = pytest.mark.gpu

RANKS = np.load(Path(__file__).resolve().parent / "golden" / "blue_noise_ranks.npy")


def _samples(data: bytes, shape: tuple[int, ...], sixteen: bool) -> np.ndarray:
    body = data.split(b"\n", 3)[3]
    values = np.frombuffer(body, dtype=">u2" if sixteen else np.uint8).astype(np.int64)
    return values.reshape(shape[0], shape[1], -1)


def test_rounding_halves_away_from_zero():
    from unround import native

    samples = np.array([[0.5, 1.5, 2.5, 254.5, 0.49999999999999994, -0.5],
                        [255.4, 255.5, 300.0, -7.0, 128.0, 1.0 / 257.0]])
    eight = native.pnm_bytes(samples, dither="none")
    header = b"P5\n6 2\n255\n"
    assert eight[: len(header)] == header
    assert list(eight[len(header):]) == [output.rounded(float(v), 1, 255) for v in samples.ravel()]
    sixteen = native.pnm_bytes(samples[:, :, np.newaxis].repeat(3, axis=2), sixteen=True, dither="none")
    header = b"P6\n6 2\n65535\n"
    assert sixteen[: len(header)] == header
    values = np.frombuffer(sixteen[len(header):], dtype=">u2")
    assert values.tolist() == [output.rounded(float(v), 257, 65535) for v in samples.ravel() for _ in range(3)]


def test_sixteen_bits_round_the_exact_product():
    from unround import native

    below = []
    for whole in range(16, 400):
        near = (whole + 0.5) / 257
        for sample in (math.nextafter(near, 0.0), near, math.nextafter(near, 256.0)):
            if sample * 257 == whole + 0.5 and Fraction(sample) * 257 < Fraction(whole + 0.5):
                below.append(sample)
    picture = np.array([below])
    data = native.pnm_bytes(picture, sixteen=True, dither="none")
    values = np.frombuffer(data[data.index(b"65535\n") + 6:], dtype=">u2")
    assert values.tolist() == [math.floor(v * 257) for v in below]


@pytest.mark.parametrize("channels", ["apart", "together"])
@pytest.mark.parametrize("sixteen", [False, True])
@pytest.mark.parametrize("shape", [(5, 7), (70, 66, 3)])
def test_the_dither_is_that_of_the_matrix(shape, channels, sixteen):
    from unround import native

    picture = np.random.default_rng(74).uniform(-3.0, 258.0, size=shape)
    picture.flat[:4] = [0.0, 255.0, 9.25, 254.75]
    data = native.pnm_bytes(picture, sixteen=sixteen, dither="blue-noise", dither_channels=channels)
    got = _samples(data, shape, sixteen)
    np.testing.assert_array_equal(got, output.levels(picture, RANKS, sixteen=sixteen, channels=channels))


def test_a_large_picture_is_dithered_as_a_small_one():
    # 1000 x 1500 RGB: every sample against the oracle's formula, vectorized in binary64 with
    # the exact error of each product (the oracle's rationals on a sample of pixels).
    from unround import native

    rng = np.random.default_rng(5)
    picture = rng.uniform(-2.0, 257.0, size=(1000, 1500, 3))
    got = _samples(native.pnm_bytes(picture), picture.shape, False)
    rows = rng.integers(0, 1000, 200)
    columns = rng.integers(0, 1500, 200)
    for i, j in zip(rows, columns):
        expected = output.levels(picture[i: i + 1, j: j + 1], np.roll(RANKS, (-i % 64, -j % 64), axis=(0, 1)),
                                 sixteen=False)
        np.testing.assert_array_equal(got[i, j], expected[0, 0], err_msg=f"pixel {i}, {j}")


def test_refusals():
    from unround import native

    with pytest.raises(native.UnroundError, match="not finite"):
        native.pnm_bytes(np.array([[np.nan]]))
    with pytest.raises(native.UnroundError, match="PNM holds no alpha"):
        native.pnm_bytes(np.zeros((2, 2, 4)))
    picture = np.full((2, 3), 7.5)
    flat = native.pnm_bytes(picture, dither="none")
    assert native.pnm_bytes(picture, dither="blue-noise", dither_channels="together") != flat
    for dither, channels in [("ordered", None), ("none", "apart"), ("blue-noise", "mixed")]:
        with pytest.raises(ValueError, match="the dither is blue-noise"):
            native.pnm_bytes(picture, dither=dither, dither_channels=channels)


@pytest.mark.parametrize("colour", [False, True])
@pytest.mark.parametrize("sixteen", [False, True])
def test_a_solve_to_levels_is_the_pnm_of_the_solve(colour, sixteen):
    # unround_b200_solve_levels quantizes the picture on the device: the levels of the binary64
    # picture that unround_solve returns, as unround_pnm makes them.
    from unround import native, synthetic

    made = (synthetic.colour(61, 83, quality=50, seed=4, noise=2) if colour
            else synthetic.grey(61, 83, quality=50, seed=4, noise=2))
    options = ["--method", "tgv", "--iterations", "20", "--tolerance", "0", "--record-every", "0"]
    picture = native.solve(made.image, options).picture
    for dither, channels in [("blue-noise", None), ("blue-noise", "together"), ("none", None)]:
        levels = native.solve_levels(made.image, options, sixteen=sixteen, dither=dither, dither_channels=channels)
        assert levels.shape == picture.shape
        expected = _samples(native.pnm_bytes(picture, sixteen=sixteen, dither=dither, dither_channels=channels),
                            picture.shape, sixteen)
        np.testing.assert_array_equal(levels.reshape(expected.shape).astype(np.int64), expected)
