"""The batched solve's host side, without a GPU: the seeded mix of pictures (sizes, layouts,
methods, qualities, alphas as the batch workload draws them), and the batch's refusals, which
come before any device work."""

import numpy as np
import pytest


def test_mix_draws():
    from unround import jpegio, synthetic

    entries = synthetic.mix(24, seed=11, smallest=32, largest=160, iterations=7)
    assert len(entries) == 24
    for e in entries:
        assert e.image.height % 16 == 0 and e.image.width % 16 == 0
        assert 32 <= e.image.height <= 160 and 32 <= e.image.width <= 160
        assert 10 <= e.quality <= 90
        assert 0.3 <= e.alpha <= 3.0
        assert e.options[e.options.index("--iterations") + 1] == "7"
        assert e.options[e.options.index("--record-every") + 1] == "0"
        if e.method == "tgv":
            alpha1 = float(e.options[e.options.index("--alpha1") + 1])
            alpha0 = float(e.options[e.options.index("--alpha0") + 1])
            assert alpha0 == pytest.approx(2 * alpha1)
        expected = jpegio.ColorSpace.YCBCR if e.colour else jpegio.ColorSpace.GRAYSCALE
        assert e.image.color_space == expected
    assert {e.method for e in entries} == {"tv", "tgv"} and {e.colour for e in entries} == {True, False}
    again = synthetic.mix(24, seed=11, smallest=32, largest=160, iterations=7)
    assert all(np.array_equal(a.image.components[0].coefficients, b.image.components[0].coefficients)
               for a, b in zip(entries, again))


def test_refusals_before_the_device():
    from unround import native, synthetic

    entries = synthetic.mix(2, seed=2, smallest=32, largest=64, iterations=5)
    images = [e.image for e in entries]
    uneven = [entries[0].options, [o if o != "5" else "6" for o in entries[1].options]]
    with pytest.raises(native.UnroundError) as caught:
        native.solve_batch(images, uneven)
    assert caught.value.status == native.Status.ARGUMENT and "same number of iterations" in str(caught.value)
    recording = [[o if o != "0" else "10" for o in e.options] for e in entries]
    with pytest.raises(native.UnroundError) as caught:
        native.solve_batch(images, recording)
    assert caught.value.status == native.Status.ARGUMENT and "--record-every 0" in str(caught.value)
    with pytest.raises(native.UnroundError) as caught:
        native.solve_batch(images, ["--method", "mmse"])
    assert caught.value.status == native.Status.OPTIONS
