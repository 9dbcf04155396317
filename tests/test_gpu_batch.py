"""The batched solve (unround_b200_solve_batch): many pictures of uneven sizes, channels,
qualities and methods solved together, each result against the same picture solved alone by
unround_solve. The batched kernels make every pixel and block by the single-picture kernels'
device functions; the compiler may fuse a multiply-add differently in the two kernels, so the
canvases agree to binary32 rounding (rel L2 <= 1e-5, max |difference| <= 1e-3 on 0..255), the
8-bit outputs on >= 99.9% of pixels, and the records' values closely."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-3


def _alone_and_batched(entries):
    from unround import native

    decoded, timing = native.solve_batch([e.image for e in entries], [e.options for e in entries])
    alone = [native.solve(e.image, e.options) for e in entries]
    return decoded, alone, timing


def _same(batched, alone, name):
    a, b = batched.canvas, alone.canvas
    assert a.shape == b.shape and np.isfinite(a).all(), name
    difference = a - b
    rel = np.linalg.norm(difference) / np.linalg.norm(b)
    assert rel <= REL_L2, f"{name}: rel L2 {rel:.3e}"
    assert np.abs(difference).max() <= MAX_ABS, f"{name}: max {np.abs(difference).max():.3e}"
    rounded = lambda x: np.clip(np.floor(x + 0.5), 0, 255)  # noqa: E731
    assert (rounded(batched.picture) == rounded(alone.picture)).mean() >= 0.999, name
    for ca, cb in zip(batched.coefficients, alone.coefficients):
        assert np.abs(ca - cb).max() <= 1e-2, name
    assert batched.result.iterations == alone.result.iterations
    assert batched.result.stop == alone.result.stop
    np.testing.assert_array_equal(batched.result.history.iterations, alone.result.history.iterations)
    np.testing.assert_allclose(batched.result.history.primal, alone.result.history.primal, rtol=1e-5, err_msg=name)
    np.testing.assert_allclose(batched.result.history.dual, alone.result.history.dual, rtol=1e-5, atol=1e-6,
                               err_msg=name)


def test_mix_equals_pictures_alone():
    from unround import synthetic

    entries = synthetic.mix(12, seed=5, smallest=48, largest=272, iterations=40)
    assert len({e.method for e in entries}) == 2 and len({e.colour for e in entries}) == 2
    decoded, alone, timing = _alone_and_batched(entries)
    assert timing.iterations == 39
    assert timing.launches_per_iteration >= 4
    assert timing.milliseconds > 0
    for n, (b, a) in enumerate(zip(decoded, alone)):
        _same(b, a, f"picture {n}: {entries[n].image.height}x{entries[n].image.width} {entries[n].method}")


def test_other_layouts_and_channels_apart():
    from unround import synthetic

    common = ["--iterations", "25", "--tolerance", "0", "--record-every", "0"]
    entries = [
        synthetic.MixEntry(synthetic.colour(40, 72, quality=60, seed=9, sampling=(1, 2)).image,
                           ["--method", "tv", "--channels", "apart", "--channel-weights", "1,0.5,0.75", *common],
                           True, "tv", 60, 1.0),
        synthetic.MixEntry(synthetic.colour(32, 40, quality=80, seed=10, sampling=(1, 1)).image,
                           ["--method", "tgv", "--centres", "mmse", "--slack", "0.5", "--slack-cost", "3", *common],
                           True, "tgv", 80, 1.0),
        synthetic.MixEntry(synthetic.grey(61, 45, quality=30, seed=4).image, ["--method", "tgv", *common],
                           False, "tgv", 30, 1.0),
        synthetic.MixEntry(synthetic.colour(61, 77, quality=75, seed=8, noise=3).image,
                           ["--method", "tgv", *common], True, "tgv", 75, 1.0),
    ]
    decoded, alone, _ = _alone_and_batched(entries)
    for n, (b, a) in enumerate(zip(decoded, alone)):
        _same(b, a, f"picture {n}")


@pytest.mark.parametrize("iterations", [1, 2, 3, 4, 5])
def test_few_iterations(iterations):
    # 1 and 2: no iteration batched or one, eagerly; 3: two, eagerly; 4: the first eagerly and one
    # launch of the graph of a pair; 5: the first, a pair, and the last of the pairs' first parity
    # eagerly.
    from unround import synthetic

    entries = synthetic.mix(3, seed=7, smallest=32, largest=96, iterations=iterations)
    decoded, alone, timing = _alone_and_batched(entries)
    assert timing.iterations == iterations - 1
    for n, (b, a) in enumerate(zip(decoded, alone)):
        _same(b, a, f"picture {n}")


def test_the_autotuner_measures_once_and_changes_no_result(monkeypatch):
    # The autotuner times each class's dual sweep at candidate tile heights before the loop
    # (launches that write only what the first iteration writes again): a batch of new shapes is
    # measured, the same shapes again are not, and the results agree with the wave model's tiles
    # and with each picture alone.
    from unround import native, synthetic

    entries = synthetic.mix(8, seed=21, smallest=64, largest=400, iterations=20)
    images, options = [e.image for e in entries], [e.options for e in entries]
    monkeypatch.setenv("UNROUND_B200_AUTOTUNE", "1")
    first, timing = native.solve_batch(images, options)
    assert timing.tuning_milliseconds > 0
    again, timing = native.solve_batch(images, options)
    assert timing.tuning_milliseconds == 0
    monkeypatch.delenv("UNROUND_B200_AUTOTUNE")
    modelled, timing = native.solve_batch(images, options)
    assert timing.tuning_milliseconds == 0
    for n, entry in enumerate(entries):
        alone = native.solve(entry.image, entry.options)
        np.testing.assert_array_equal(first[n].canvas, again[n].canvas)
        _same(first[n], alone, f"picture {n} tuned")
        _same(modelled[n], alone, f"picture {n} modelled")
