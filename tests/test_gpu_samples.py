"""Pictures of rounded samples reconstructed on the GPU (unround_b200_solve_samples) against the
reference's own solver of them (cpp/src/samples.cpp through the oracle's bridge), on the same
levels and options after a fixed number of iterations: relative L2 <= 1e-4 and max |difference|
<= 2e-3 on the 0-255 scale, every sample of the result within its interval in binary64, and the
records' gap within 1e-3 of the reference's (relative); the defaults of PNG files (tolerance
1e-4, TGV's ratio 0.3) stop both near the same picture; 8 and 16 bits, grey, RGB and an alpha apart;
and rounded back without a dither, an 8-bit result gives back its levels."""

from pathlib import Path

import numpy as np
import pytest

from oracle import output, reference

pytestmark = pytest.mark.gpu


def _picture(rows: int, columns: int, channels: int, bits: int, seed: int) -> np.ndarray:
    """Levels of a smooth picture with a few edges: ramps, a disc and a gentle wave per channel."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:rows, 0:columns].astype(np.float64)
    top = 2**bits - 1
    planes = []
    for c in range(channels):
        base = rng.uniform(30, 200) + rng.uniform(-1.5, 1.5) * x + rng.uniform(-1.5, 1.5) * y
        disc = ((y - rows * rng.uniform(0.3, 0.7)) ** 2 + (x - columns * rng.uniform(0.3, 0.7)) ** 2) < (rows / 4) ** 2
        value = base + 40 * disc + 6 * np.sin(x / rng.uniform(4, 9))
        planes.append(np.clip(value, 0, 255) * top / 255)
    return np.rint(np.stack(planes, -1)).astype(np.uint16)


CASES = [
    ("grey-tgv-8", (40, 56, 1), 8, ["--method", "tgv"]),
    ("rgb-tv-mu-8", (36, 48, 3), 8, ["--method", "tv", "--alpha", "1.5", "--mu", "0.05"]),
    ("grey-tgv-16", (32, 40, 1), 16, ["--method", "tgv", "--alpha1", "2", "--alpha0", "4"]),
    ("rgba-tgv-8", (30, 44, 4), 8, ["--method", "tgv"]),
    ("grey-tv-slack-8", (34, 38, 1), 8, ["--method", "tv", "--slack", "0.25", "--mu", "0.01"]),
]


@pytest.mark.parametrize("name, shape, bits, options", CASES, ids=[c[0] for c in CASES])
def test_against_the_reference_solver(name, shape, bits, options):
    from unround import native

    levels = _picture(*shape, bits, seed=len(name))
    fixed = [*options, "--iterations", "150", "--tolerance", "0", "--record-every", "50"]
    ours = native.solve_samples(levels, bits, fixed)
    theirs = reference.solve_samples(levels, bits, fixed)
    got = ours.canvas.reshape(theirs.canvas.shape)
    assert np.linalg.norm(got - theirs.canvas) / np.linalg.norm(theirs.canvas) <= 1e-4, name
    assert np.abs(got - theirs.canvas).max() <= 2e-3, name
    # Within the intervals, in binary64.
    slack = float(options[options.index("--slack") + 1]) if "--slack" in options else 0.0
    ends = np.array([[native_interval(int(v), bits, slack) for v in plane.ravel()]
                     for plane in np.moveaxis(levels, -1, 0)])
    flat = got.reshape(got.shape[0], -1)
    assert np.all(flat >= ends[..., 0]) and np.all(flat <= ends[..., 1]), name
    # The records: the same iterations, the gap alike.
    history = ours.result.history
    np.testing.assert_array_equal(history.iterations, theirs.record_iterations)
    gap_ours = history.primal - history.dual
    gap_theirs = theirs.records[:, 1] - theirs.records[:, 2]
    assert np.all(np.abs(gap_ours - gap_theirs) <= 1e-3 * np.abs(theirs.records[:, 1]) + 1e-6), (name, gap_ours, gap_theirs)
    # The picture interleaves the planes.
    np.testing.assert_array_equal(ours.picture.reshape(shape[0], shape[1], -1), np.moveaxis(got, 0, -1))


def native_interval(level: int, bits: int, slack: float = 0.0) -> tuple[float, float]:
    import ctypes

    from unround import native

    library = native._library()
    library.unround_b200_sample_interval.restype = ctypes.c_int32
    library.unround_b200_sample_interval.argtypes = [ctypes.c_uint32, ctypes.c_int32, ctypes.c_double,
                                                     ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_size_t]
    ends = (ctypes.c_double * 3)()
    assert library.unround_b200_sample_interval(level, bits, slack, ends, None, 0) == 0
    return ends[0], ends[1]


def test_the_defaults_of_png_files():
    from unround import native

    levels = _picture(28, 36, 3, 8, seed=3)
    ours = native.solve_samples(levels, 8, ["--method", "tgv", "--iterations", "3"])
    theirs = reference.solve_samples(levels, 8, ["--method", "tgv", "--iterations", "3"])
    assert ours.result.iterations == theirs.iterations == 3
    # Stopped by the default tolerance of PNG files, as the reference stops.
    ours = native.solve_samples(levels, 8, ["--method", "tgv", "--record-every", "10"])
    theirs = reference.solve_samples(levels, 8, ["--method", "tgv", "--record-every", "10"])
    assert theirs.stop == 1 and int(ours.result.stop) == 1
    # A gap per sample of 1e-4 is near what binary32 iterates resolve on the 0-255 scale: the
    # device stops within half again the reference's iterations, at the same picture.
    assert ours.result.iterations <= 1.5 * theirs.iterations + 50
    got = ours.canvas.reshape(theirs.canvas.shape)
    assert np.linalg.norm(got - theirs.canvas) / np.linalg.norm(theirs.canvas) <= 1e-4


def test_an_eight_bit_result_gives_back_its_levels():
    from unround import native

    levels = _picture(40, 48, 3, 8, seed=9)
    ours = native.solve_samples(levels, 8, ["--method", "tgv", "--iterations", "200", "--tolerance", "0"])
    rounded = np.frombuffer(native.pnm_bytes(ours.picture, dither="none").split(b"\n", 3)[3], dtype=np.uint8)
    np.testing.assert_array_equal(rounded.reshape(levels.shape), levels)


def test_refusals():
    from unround import native

    levels = _picture(8, 8, 1, 8, seed=1)
    with pytest.raises(native.UnroundError, match="not for a PNG file"):
        native.solve_samples(levels, 8, ["--method", "tgv", "--mu-scale", "3"])
    with pytest.raises(native.UnroundError, match="tv or tgv"):
        native.solve_samples(levels, 8, ["--method", "mmse"])
    with pytest.raises(native.UnroundError, match="bits are not taken"):
        native.solve_samples(levels, 17, ["--method", "tgv"])
    with pytest.raises(native.UnroundError, match="below 2"):
        native.solve_samples(np.full((4, 4), 300, dtype=np.uint16), 8, ["--method", "tgv"])


def test_the_measured_loop():
    """unround_b200_measure_samples times the loop of the same solver: its counts are the
    picture's, both kernels took time, and a colour picture with an alpha is refused."""
    from unround import native

    levels = _picture(64, 96, 3, 8, seed=4)
    timing = native.measure_samples(levels, 8, ["--method", "tgv"], warmup=3, iterations=20)
    assert timing.iterations == 20 and timing.pixels == 64 * 96 and timing.samples == 3 * 64 * 96
    assert timing.launches_per_iteration == 2
    assert timing.milliseconds > 0 and timing.dual_milliseconds > 0 and timing.primal_milliseconds > 0
    with pytest.raises(native.UnroundError):
        native.measure_samples(_picture(8, 8, 4, 8, seed=1), 8, ["--method", "tgv"])


@pytest.mark.parametrize("shape, options", [
    ((45, 61, 3), ["--method", "tgv"]),
    ((37, 29, 1), ["--method", "tv", "--mu", "0.05"]),
    ((52, 70, 3), ["--method", "tv", "--channels", "apart"]),
    ((19, 100, 3), ["--method", "tgv", "--channels", "apart", "--slack", "0.3"]),
])
def test_the_fused_sweeps_equal_the_two_launches(monkeypatch, shape, options):
    """The samples' primal step inside the dual sweep (UNROUND_B200_KERNELS=sweep) and in the
    fused sweep of iteration.cu (=fused), one launch an iteration each, against the dual sweep and
    the primal kernel apart (the default), on ragged sizes: the same iterations, the canvases to
    binary32 rounding."""
    from unround import native

    levels = _picture(*shape, 8, seed=shape[0])
    given = [*options, "--iterations", "90", "--tolerance", "0"]
    launches = {}
    made = {}
    for mode in ("split", "fused", "sweep", None):
        if mode is None:
            monkeypatch.delenv("UNROUND_B200_KERNELS", raising=False)
        else:
            monkeypatch.setenv("UNROUND_B200_KERNELS", mode)
        made[mode] = native.solve_samples(levels, 8, given)
        launches[mode] = native.measure_samples(levels, 8, options, warmup=2, iterations=5).launches_per_iteration
    assert launches == {"split": 2, "fused": 1, "sweep": 1, None: 2}
    split = made["split"]
    np.testing.assert_array_equal(made[None].canvas, split.canvas)
    for mode in ("fused", "sweep"):
        assert made[mode].result.iterations == split.result.iterations == 90
        difference = made[mode].canvas - split.canvas
        assert np.linalg.norm(difference) / np.linalg.norm(split.canvas) <= 1e-5, mode
        assert np.abs(difference).max() <= 1e-3, mode
