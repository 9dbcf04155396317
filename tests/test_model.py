"""The host model (binary64 setup of the path) against the reference's own C++ solver, without a
GPU: interval ends, weights, steps, flat blocks and tau/sigma to the last bit; MMSE centres within
(2|q| + 20) u Q of the reference's (docs/math.md 9.2); the refusals of inputs the reference refuses."""

import numpy as np
import pytest

from oracle import reference
from unround import jpegio, native, synthetic

pytestmark = pytest.mark.skipif(not reference.available(), reason="oracle/_ref is not built (make -C oracle/ref)")


def _theirs(image, options):
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor) for c in image.components]
    return reference.solve(image.height, image.width, int(image.color_space), components, options)


CASES = [
    ("grey-default-tgv", lambda: synthetic.grey(45, 61, quality=50, seed=1).image, ["--method", "tgv", "--iterations", "0"]),
    ("grey-tv-mmse", lambda: synthetic.grey(64, 64, quality=30, seed=2).image,
     ["--method", "tv", "--centres", "mmse", "--iterations", "0"]),
    ("grey-slack-power", lambda: synthetic.grey(32, 40, quality=70, seed=3).image,
     ["--method", "tv", "--slack", "0.25", "--slack-cost", "2", "--weight-power", "1.5", "--dc-weight", "0.5",
      "--flat-levels", "3", "--flat-dc", "any", "--iterations", "0"]),
    ("colour420-rule", lambda: synthetic.colour(48, 80, quality=75, seed=4).image,
     ["--method", "tgv", "--alpha1", "0.7", "--alpha0", "1.3", "--iterations", "0"]),
    ("colour422-mu-list", lambda: synthetic.colour(40, 64, quality=60, seed=5, sampling=(1, 2)).image,
     ["--method", "tv", "--mu", "0.5,rule,0.01", "--mu-power", "1", "--channel-weights", "1,0.5,0.25", "--iterations", "0"]),
]


@pytest.mark.parametrize("name,make,options", CASES, ids=[c[0] for c in CASES])
def test_model_matches_reference(name, make, options):
    image = make()
    theirs = _theirs(image, options)
    for index, component in enumerate(image.components):
        shape = component.coefficients.shape
        np.testing.assert_array_equal(native.model(image, options, index, 0).reshape(shape), theirs.lower[index])
        np.testing.assert_array_equal(native.model(image, options, index, 1).reshape(shape), theirs.upper[index])
        ours_centres = native.model(image, options, index, 2).reshape(shape)
        q = component.coefficients.astype(np.float64)
        steps = component.quant_table.reshape(8, 8).astype(np.float64)
        bound = (2 * np.abs(q) + 20) * 2.0**-53 * steps
        assert np.all(np.abs(ours_centres - theirs.centres[index]) <= bound)
        np.testing.assert_array_equal(native.model(image, options, index, 4).reshape(8, 8), theirs.weights[index])
        np.testing.assert_array_equal(native.model(image, options, index, 5).reshape(8, 8), theirs.flat_weights[index])
        flat = native.model(image, options, index, 6).reshape(theirs.flat[index].shape)
        np.testing.assert_array_equal(flat.astype(np.uint8), theirs.flat[index])
    plan = native.model(image, options, 0, 7)
    # tau and sigma of a 1-iteration solve of the reference.
    once = [o if o != "0" or options[i - 1] != "--iterations" else "1" for i, o in enumerate(options)]
    ran = _theirs(image, once)
    assert (plan[0], plan[1]) == (ran.tau, ran.sigma)


def test_refusals_of_inputs():
    good = synthetic.colour(32, 32, quality=50, seed=6).image
    # Sampling factors that do not divide the largest.
    c = good.components
    bad = jpegio.image_of(32, 32, 2, [(c[0].coefficients, c[0].quant_table, 3, 2), (c[1].coefficients, c[1].quant_table, 2, 1),
                                      (c[2].coefficients, c[2].quant_table, 1, 1)])
    with pytest.raises(native.UnroundError) as raised:
        native.model(bad, ["--method", "tv"])
    assert raised.value.status == native.Status.UNSUPPORTED
    # A quantization step of 0.
    zero = good.components[0].quant_table.copy()
    zero[0, 0] = 0
    grey = jpegio.image_of(32, 32, 1, [(good.components[0].coefficients, zero, 1, 1)])
    with pytest.raises(native.UnroundError) as raised:
        native.model(grey, ["--method", "tv"])
    assert raised.value.status == native.Status.OPTIONS
    # A colour space without its components.
    with pytest.raises(native.UnroundError) as raised:
        native.model(jpegio.image_of(32, 32, 2, [(good.components[0].coefficients, good.components[0].quant_table, 1, 1)]),
                     ["--method", "tv"])
    assert raised.value.status == native.Status.UNSUPPORTED


@pytest.mark.parametrize("height, width, rows", [(0, 32, 4), (32, 0, 4), (32, 32, 2), (40, 32, 4), (32, 32, 0)],
                         ids=["no-rows", "no-columns", "blocks-short", "picture-taller", "no-blocks"])
def test_refusals_of_empty_and_ragged_inputs(height, width, rows):
    """A picture without samples, or blocks that do not cover it, is refused before any device
    work, as the reference's solver refuses it."""
    good = synthetic.grey(32, 32, quality=50, seed=6).image
    c = good.components[0]
    blocks = np.ascontiguousarray(c.coefficients[:rows]) if rows else np.zeros((0, 4, 8, 8), np.int16)
    image = jpegio.image_of(height, width, 1, [(blocks, c.quant_table, 1, 1)])
    with pytest.raises(native.UnroundError) as raised:
        native.model(image, ["--method", "tv"])
    assert raised.value.status == native.Status.UNSUPPORTED
    with pytest.raises(Exception):
        _theirs(image, ["--method", "tv", "--iterations", "0"])


def test_reused_host_blocks_leave_no_trace():
    """The model's levels and flat flags come from host blocks that earlier calls have used: the
    same picture gives the same arrays before and after others, larger and smaller."""
    options = ["--method", "tgv", "--flat-levels", "2", "--flat-dc", "3", "--iterations", "0"]
    first = synthetic.grey(96, 80, quality=40, seed=31).image
    before = [native.model(first, options, 0, which) for which in (0, 1, 2, 6)]
    for seed, size in ((32, (200, 160)), (33, (24, 40)), (34, (120, 136))):
        native.model(synthetic.grey(*size, quality=70, seed=seed).image, options, 0, 6)
    after = [native.model(first, options, 0, which) for which in (0, 1, 2, 6)]
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a, b)
