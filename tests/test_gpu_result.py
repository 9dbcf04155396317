"""The result of a solve as the C interface hands it over: the planes are the canvas cut to the
picture, and the picture is the planes' JFIF RGB (YCbCr), the planes interleaved, or the one
plane -- made on the device, bit for bit what the host's unround_to_rgb and a crop make of the
canvas (rust/unround/src/decode.rs:306-364); repeated calls reuse the pinned result blocks."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPTIONS = ["--method", "tgv", "--iterations", "5", "--tolerance", "0", "--record-every", "0"]


@pytest.mark.parametrize("rows, columns", [(61, 77), (64, 96)])
def test_colour_picture_is_the_rgb_of_the_cut_canvas(rows, columns):
    from unround import native, synthetic

    image = synthetic.colour(rows, columns, quality=60, seed=rows, noise=2).image
    decoded = native.solve(image, OPTIONS)
    cut = decoded.canvas[:, :rows, :columns]
    np.testing.assert_array_equal(decoded.planes, cut)
    np.testing.assert_array_equal(decoded.picture, native.to_rgb(cut))


@pytest.mark.parametrize("rows, columns", [(45, 50), (48, 64)])
def test_grey_picture_is_the_cut_canvas(rows, columns):
    from unround import native, synthetic

    image = synthetic.grey(rows, columns, quality=60, seed=rows, noise=2).image
    decoded = native.solve(image, OPTIONS)
    np.testing.assert_array_equal(decoded.planes, decoded.canvas[:, :rows, :columns])
    np.testing.assert_array_equal(decoded.picture, decoded.canvas[0, :rows, :columns])


def test_repeated_calls_give_the_same_result():
    from unround import native, synthetic

    image = synthetic.colour(96, 80, quality=50, seed=3, noise=2).image
    first = native.solve(image, OPTIONS)
    for _ in range(3):
        again = native.solve(image, OPTIONS)
        np.testing.assert_array_equal(again.picture, first.picture)
        np.testing.assert_array_equal(again.canvas, first.canvas)
        for a, b in zip(again.coefficients, first.coefficients):
            np.testing.assert_array_equal(a, b)


def test_decoder_of_the_centres_has_the_picture_too():
    from unround import native, synthetic

    image = synthetic.colour(40, 56, quality=40, seed=9).image
    decoded = native.solve(image, ["--method", "mmse"])
    cut = decoded.canvas[:, :40, :56]
    np.testing.assert_array_equal(decoded.picture, native.to_rgb(cut))
