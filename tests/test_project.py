"""A picture made elsewhere projected onto a JPEG file's intervals (unround_project; docs/math.md 12
of the reference), on the host in binary64, against the reference's own projection
(cpp/src/picture.cpp through the oracle's bridge) on the same file and picture: the projected
canvas, the clipped coefficients and the excess within 1e-9 (binary64 rounding: the DCTs' sums
in another order); grey and 4:2:0/4:2:2/4:4:4 colour, with a slack. A projection projected again
lies within the intervals (a picture of whole MCUs); pictures of the wrong size, or not finite,
are refused. No GPU is needed."""

import io

import numpy as np
import pytest
from PIL import Image as PILImage

from oracle import reference
from unround import jpegio, native


def _file(mode: str, subsampling: int, shape: tuple[int, int], seed: int, quality: int = 50):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0 : shape[0], 0 : shape[1]]
    base = np.clip(128 + 60 * np.sin(x / 7) * np.cos(y / 5) + rng.normal(0, 6, shape), 0, 255)
    picture = base if mode == "L" else np.stack([base, np.roll(base, 3, 1), 255 - base], -1)
    buffer = io.BytesIO()
    PILImage.fromarray(picture.astype(np.uint8)).save(buffer, format="JPEG", quality=quality, subsampling=subsampling)
    # The picture made elsewhere: the original samples with a little noise of their own.
    return buffer.getvalue(), picture + rng.normal(0, 1.5, picture.shape)


CASES = [("L", 0, (45, 70), []), ("RGB", 2, (45, 70), []), ("RGB", 1, (33, 50), ["--slack", "0.25"]),
         ("RGB", 0, (40, 24), [])]


@pytest.mark.parametrize("mode, subsampling, shape, extra", CASES, ids=[f"{c[0]}-{c[1]}" for c in CASES])
def test_against_the_reference_projection(mode, subsampling, shape, extra):
    data, picture = _file(mode, subsampling, shape, seed=subsampling + len(extra))
    options = ["--method", "tv", *extra]
    ours = native.project(picture, data, options)
    image = jpegio.read(data)
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor)
                  for c in image.components]
    theirs = reference.project(image.height, image.width, int(image.color_space), components, options, picture)
    assert ours.result is None and ours.input_format == "jpeg"
    np.testing.assert_allclose(ours.canvas, theirs.canvas, rtol=0, atol=1e-9)
    for mine, other in zip(ours.coefficients, theirs.coefficients):
        np.testing.assert_allclose(mine, other, rtol=0, atol=1e-9)
    for mine, other in zip(ours.excess, theirs.excess):
        np.testing.assert_allclose(mine, other, rtol=0, atol=1e-10)
    assert sum(int((e > 0).sum()) for e in ours.excess) > 0  # the noise put some outside
    for problem, coefficients in zip(ours.problems, ours.coefficients):
        assert np.all(coefficients >= problem.lower) and np.all(coefficients <= problem.upper)


def test_a_projection_projected_again_lies_within():
    data, picture = _file("RGB", 2, (48, 64), seed=7)
    once = native.project(picture, data, ["--method", "tv"])
    twice = native.project(once.picture, data, ["--method", "tv"])
    assert max(float(e.max()) for e in twice.excess) <= 1e-9
    np.testing.assert_allclose(twice.canvas, once.canvas, rtol=0, atol=1e-9)


def test_refusals():
    data, picture = _file("L", 0, (16, 24), seed=1)
    with pytest.raises(native.UnroundError) as raised:
        native.project(picture[:8], data, ["--method", "tv"])
    assert raised.value.status == native.Status.OPTIONS
    bad = picture.copy()
    bad[3, 4] = np.nan
    with pytest.raises(native.UnroundError) as raised:
        native.project(bad, data, ["--method", "tv"])
    assert raised.value.status == native.Status.OPTIONS
    with pytest.raises(native.UnroundError) as raised:
        native.project(picture, b"not a file", ["--method", "tv"])
    assert raised.value.status == native.Status.READ
