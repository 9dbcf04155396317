"""The observer of a solve (unround.h's unround_observer; the reference's Python observer,
python/src/unround/native.py solve/decode): called after every record but the first with the
record's iteration, values and canvas; a true return stops the solve there (Stop 3, OBSERVER)
with that record's canvas as the result; an exception it raises stops the solve and is raised by
the call that ran it; the decoder of the centres has no records and calls it never."""

import io
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _identical(a: float, b: float) -> bool:
    return struct.pack("<d", a) == struct.pack("<d", b)


def _bits(values) -> np.ndarray:
    return np.ascontiguousarray(values, dtype=np.float64).view(np.uint64)


def _colour_file() -> bytes:
    from PIL import Image

    from unround import synthetic

    rgb = np.clip(synthetic.colour(45, 62, quality=50, seed=31, noise=2).samples, 0, 255).astype(np.uint8)
    stream = io.BytesIO()
    Image.fromarray(rgb).save(stream, format="JPEG", quality=40, subsampling=2)
    return stream.getvalue()


@pytest.mark.parametrize("source", ["arrays", "file"])
def test_observer_sees_the_records_and_stops_the_solve(source):
    from unround import native, synthetic
    from unround.settings import PdhgOptions, Settings

    seen = []

    def observer(record) -> bool:
        seen.append(record)
        return record.iteration >= 10

    settings = Settings(method="tgv", pdhg=PdhgOptions(iterations=100, tolerance=0.0, record_every=5))
    if source == "arrays":
        decoded = native.solve(synthetic.colour(45, 62, quality=50, seed=31, noise=2).image, settings, observer=observer)
    else:
        decoded = native.decode(_colour_file(), settings, observer=observer)
    assert decoded.result is not None
    assert decoded.result.stop is native.Stop.OBSERVER
    assert decoded.result.iterations == 10
    history = decoded.result.history
    assert history.iterations.tolist() == [0, 5, 10]
    assert [record.iteration for record in seen] == [5, 10]
    for index, record in enumerate(seen, start=1):
        assert _identical(record.primal, float(history.primal[index]))
        assert _identical(record.dual, float(history.dual[index]))
        assert record.canvas.shape == decoded.canvas.shape
        assert np.isfinite(record.canvas).all()
    # The solve stopped at the last record: its canvas is the result's, to the last bit.
    np.testing.assert_array_equal(_bits(seen[-1].canvas), _bits(decoded.canvas))
    # The canvas an observer sees moves from record to record.
    assert not np.array_equal(seen[0].canvas, seen[1].canvas)


def test_observer_that_never_stops_changes_nothing():
    from unround import native, synthetic

    image = synthetic.grey(40, 56, quality=30, seed=32).image
    options = ["--method", "tv", "--iterations", "30", "--tolerance", "0", "--record-every", "10"]
    seen = []
    watched = native.solve(image, options, observer=lambda record: seen.append(record.iteration) and False)
    alone = native.solve(image, options)
    assert seen == [10, 20, 30]
    assert watched.result.stop is native.Stop.ITERATIONS
    np.testing.assert_array_equal(_bits(watched.canvas), _bits(alone.canvas))
    np.testing.assert_array_equal(_bits(watched.result.history.primal), _bits(alone.result.history.primal))


def test_observer_exception_stops_the_solve_and_is_raised():
    from unround import native, synthetic
    from unround.settings import PdhgOptions, Settings

    calls = 0

    def observer(record) -> bool:
        nonlocal calls
        calls += 1
        raise LookupError(f"stopped at {record.iteration}")

    settings = Settings(method="tv", pdhg=PdhgOptions(iterations=1000, tolerance=0.0, record_every=1))
    with pytest.raises(LookupError, match="stopped at 1"):
        native.solve(synthetic.grey(32, 40, quality=30, seed=33).image, settings, observer=observer)
    assert calls == 1


def test_decoder_of_the_centres_calls_no_observer():
    from unround import native, synthetic
    from unround.settings import Settings

    seen = []
    decoded = native.solve(synthetic.grey(32, 40, quality=30, seed=34).image, Settings(method="mmse"),
                           observer=lambda record: seen.append(record) or False)
    assert decoded.result is None
    assert seen == []
