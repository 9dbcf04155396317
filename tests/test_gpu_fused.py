"""The fused iteration sweep (one launch: the dual step and the next primal step) against the
split kernels (dual, then primal per component) on the same inputs and options: the same
arithmetic but for the order of the 8x8 transforms' sums, so the canvases agree to binary32
rounding (rel L2 <= 1e-5, max |difference| <= 1e-3 on 0..255), the 8-bit outputs nearly
everywhere, and the records' primal values closely. UNROUND_B200_KERNELS=fused selects the fused
sweep; the split kernels are the default."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-3


def _solve(image, options, split):
    from unround import native

    if split:
        os.environ.pop("UNROUND_B200_KERNELS", None)
    else:
        os.environ["UNROUND_B200_KERNELS"] = "fused"
    try:
        return native.solve(image, options)
    finally:
        os.environ.pop("UNROUND_B200_KERNELS", None)


def _cases():
    from unround import synthetic

    base = ["--tolerance", "0", "--record-every", "25"]
    yield "grey-tv", lambda: synthetic.grey(96, 80, quality=50, seed=3).image, ["--method", "tv", "--iterations", "100", *base]
    yield "grey-tgv-ragged", lambda: synthetic.grey(61, 45, quality=30, seed=4).image, ["--method", "tgv", "--iterations", "100", *base]
    yield "grey-tgv-tall", lambda: synthetic.grey(600, 72, quality=40, seed=11, noise=2).image, [
        "--method", "tgv", "--iterations", "60", *base]
    yield "colour420-tgv", lambda: synthetic.colour(61, 77, quality=75, seed=8, noise=3).image, [
        "--method", "tgv", "--iterations", "80", *base]
    yield "colour420-tgv-tall", lambda: synthetic.colour(560, 112, quality=60, seed=12, noise=3).image, [
        "--method", "tgv", "--iterations", "50", *base]
    yield "colour422-tv-apart", lambda: synthetic.colour(40, 72, quality=60, seed=9, sampling=(1, 2)).image, [
        "--method", "tv", "--iterations", "60", "--channels", "apart", "--channel-weights", "1,0.5,0.75", *base]
    yield "colour440-tgv", lambda: synthetic.colour(48, 40, quality=60, seed=13, sampling=(2, 1)).image, [
        "--method", "tgv", "--iterations", "60", *base]
    yield "colour444-tgv-mmse-slack", lambda: synthetic.colour(32, 40, quality=80, seed=10, sampling=(1, 1)).image, [
        "--method", "tgv", "--iterations", "60", "--centres", "mmse", "--slack", "0.5", "--slack-cost", "3", *base]
    yield "colour420-tv-512", lambda: synthetic.colour(512, 512, quality=50, seed=14, noise=2).image, [
        "--method", "tv", "--iterations", "100", "--tolerance", "0", "--record-every", "0"]


CASES = list(_cases())


@pytest.mark.parametrize("name,make,options", CASES, ids=[c[0] for c in CASES])
def test_fused_against_split(name, make, options):
    image = make()
    fused = _solve(image, options, split=False)
    split = _solve(image, options, split=True)
    a, b = fused.canvas, split.canvas
    assert a.shape == b.shape
    assert np.isfinite(a).all()
    difference = a - b
    rel = np.linalg.norm(difference) / np.linalg.norm(b)
    assert rel <= REL_L2, f"{name}: rel L2 {rel:.3e}"
    assert np.abs(difference).max() <= MAX_ABS, f"{name}: max {np.abs(difference).max():.3e}"
    rounded = lambda x: np.clip(np.floor(x + 0.5), 0, 255)  # noqa: E731
    assert (rounded(a) == rounded(b)).mean() >= 0.999
    assert fused.result.iterations == split.result.iterations
    ha, hb = fused.result.history, split.result.history
    np.testing.assert_array_equal(ha.iterations, hb.iterations)
    np.testing.assert_allclose(ha.primal, hb.primal, rtol=1e-5)
    for ca, cb in zip(fused.coefficients, split.coefficients):
        assert np.abs(ca - cb).max() <= 1e-2
