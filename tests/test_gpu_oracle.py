"""The CUDA path against the reference's own C++ solver (oracle/_ref) on the same seeded inputs
and the same option strings, through the C interface: relative L2 <= 1e-4 and max |difference|
<= 2e-3 of the canvas, the 8-bit output identical on >= 99.9% of pixels, every record (primal
and dual values, TGV's scaling and partial gap) within 1e-4 of the reference's relative to the
record's scale, the same stop, and every coefficient within its interval in binary64."""

import numpy as np
import pytest

from conftest import canvas_figures, report_parity
from oracle import reference

pytestmark = pytest.mark.gpu

REL_L2 = 1e-4
MAX_ABS = 2e-3
RECORDS = 1e-4


def _rounded(picture: np.ndarray) -> np.ndarray:
    """8-bit output: the nearest level, halves away from 0, clamped (docs/math.md 10)."""
    return np.clip(np.sign(picture) * np.floor(np.abs(picture) + 0.5), 0, 255)


def record_differences(history, record_iterations, records) -> dict[str, float]:
    """The largest differences of the device's records from the reference's (columns: seconds,
    primal, dual, scaling, partial gap): the values relative to the record's scale
    max(|P|, |D|), the scaling relative to itself. The same iterations and the same records left
    undefined (NaN) are asserted here."""
    assert list(history.iterations) == list(record_iterations)
    scale = np.maximum(np.abs(records[:, 1]), np.abs(records[:, 2]))
    worst = {}
    columns = (("primal", history.primal, 1, scale), ("dual", history.dual, 2, scale),
               ("scaling", history.scaling, 3, None), ("partial_gap", history.partial_gap, 4, scale))
    for name, ours, column, by in columns:
        ours, theirs = np.asarray(ours, dtype=np.float64), np.asarray(records[:, column], dtype=np.float64)
        assert np.array_equal(np.isnan(ours), np.isnan(theirs)), (name, ours, theirs)
        known = ~np.isnan(theirs)
        denominator = np.abs(theirs[known]) if by is None else by[known]
        difference = np.abs(ours[known] - theirs[known]) / np.maximum(denominator, 1e-300)
        worst[name] = float(difference.max()) if difference.size else 0.0
    return worst


def rounded_match(ours_picture: np.ndarray, theirs_canvas: np.ndarray, image) -> float:
    """The share of 8-bit output samples of the picture that are identical."""
    from unround import native

    if image.color_space == 2:
        theirs_picture = native.to_rgb(theirs_canvas[:, : image.height, : image.width])
    else:
        theirs_picture = np.moveaxis(theirs_canvas[:, : image.height, : image.width], 0, -1).squeeze()
    return float(np.mean(_rounded(ours_picture) == _rounded(theirs_picture)))


def _oracle(image, options):
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor) for c in image.components]
    return reference.solve(image.height, image.width, int(image.color_space), components, options)


def _cases():
    from unround import synthetic

    base = ["--tolerance", "0"]
    yield "grey-tv-ragged", lambda: synthetic.grey(61, 45, quality=50, seed=3).image, ["--method", "tv", "--iterations", "100", *base]
    yield "grey-tgv", lambda: synthetic.grey(64, 48, quality=30, seed=4).image, ["--method", "tgv", "--iterations", "100", *base]
    yield "grey-tgv-one-block", lambda: synthetic.grey(8, 8, quality=50, seed=5).image, ["--method", "tgv", "--iterations", "30", *base]
    yield "grey-tv-one-row", lambda: synthetic.grey(8, 64, quality=50, seed=6).image, ["--method", "tv", "--iterations", "40", *base]
    yield "grey-tv-mmse-slack", lambda: synthetic.grey(40, 56, quality=40, seed=7).image, [
        "--method", "tv", "--iterations", "60", "--centres", "mmse", "--slack", "0.5", "--slack-cost", "3", *base]
    yield "colour420-tgv", lambda: synthetic.colour(61, 77, quality=75, seed=8, noise=3).image, [
        "--method", "tgv", "--iterations", "60", *base]
    yield "colour422-tv-apart", lambda: synthetic.colour(40, 72, quality=60, seed=9, sampling=(1, 2)).image, [
        "--method", "tv", "--iterations", "50", "--channels", "apart", "--channel-weights", "1,0.5,0.75", *base]
    yield "colour444-tgv-partial", lambda: synthetic.colour(32, 40, quality=80, seed=10, sampling=(1, 1)).image, [
        "--method", "tgv", "--iterations", "40", "--partial-radius", "20", *base]
    yield "config1-tv-512", lambda: synthetic.grey(512, 512, quality=50, seed=1).image, [
        "--method", "tv", "--alpha", "1", "--iterations", "200", "--tolerance", "0", "--record-every", "0",
        "--step-ratio", "1", "--step-product", "0.99", "--norm-squared", "7.92"]
    yield "config2-tgv-colour-reduced", lambda: synthetic.colour(240, 320, quality=75, seed=2, noise=3).image, [
        "--method", "tgv", "--alpha1", "1", "--alpha0", "2", "--iterations", "100", "--tolerance", "0", "--record-every", "50"]
    rng = np.random.default_rng(5)
    steps = rng.integers(1, 65, size=64)
    yield "config5-tgv-custom-reduced", lambda: synthetic.grey(256, 256, seed=5, noise=2, steps=steps).image, [
        "--method", "tgv", "--alpha1", "1.5", "--alpha0", "3", "--iterations", "100", "--tolerance", "0", "--record-every", "50"]


CASES = list(_cases())


@pytest.mark.parametrize("name,make,options", CASES, ids=[c[0] for c in CASES])
def test_against_reference(name, make, options):
    from unround import native

    image = make()
    ours = native.solve(image, options)
    theirs = _oracle(image, options)
    assert ours.canvas.shape == theirs.canvas.shape
    figures = canvas_figures(ours.canvas, theirs.canvas)
    same = rounded_match(ours.picture, theirs.canvas, image)
    worst = record_differences(ours.result.history, theirs.record_iterations, theirs.records)
    report_parity(name, **figures, same_8bit=same, **{f"record_{k}": v for k, v in worst.items()})
    assert figures["rel_l2"] <= REL_L2, figures
    assert figures["max_abs"] <= MAX_ABS, figures
    assert same >= 0.999, same
    assert max(worst.values()) <= RECORDS, worst
    assert ours.result.iterations == theirs.iterations
    # Intervals bit for bit; every coefficient within them.
    for index, problem in enumerate(ours.problems):
        np.testing.assert_array_equal(problem.lower, theirs.lower[index])
        np.testing.assert_array_equal(problem.upper, theirs.upper[index])
        np.testing.assert_array_equal(problem.weights, theirs.weights[index])
        c = ours.coefficients[index]
        assert np.all(c >= problem.lower) and np.all(c <= problem.upper)
