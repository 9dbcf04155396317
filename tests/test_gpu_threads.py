"""Calls from several threads at once (rust/capi/include/unround.h:22-24; the reference's
python/tests/test_native.py:478-494): each call has its own CUDA stream and device buffers, and
the host state the calls share (the pinned-buffer cache, the dither's ranks on the device, the
launchers' set-up) is safe to share, so files reconstructed from four threads at once come out
bit for bit as they do one at a time."""

import io
import threading

import numpy as np
import pytest
from PIL import Image as PILImage

pytestmark = pytest.mark.gpu


def _file(seed: int, shape: tuple[int, ...], format: str, **options: object) -> bytes:
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0 : shape[0], 0 : shape[1]].astype(np.float64)
    layers = [np.clip(128 + 70 * np.sin(x / (6 + c) + y / 9) + rng.normal(0, 4, shape[:2]), 0, 255)
              for c in range(shape[2] if len(shape) == 3 else 1)]
    pixels = np.rint(np.stack(layers, -1)).astype(np.uint8)
    buffer = io.BytesIO()
    PILImage.fromarray(pixels[..., 0] if len(shape) == 2 else pixels).save(buffer, format=format, **options)
    return buffer.getvalue()


def test_threads_reconstruct_at_once():
    from unround import native

    files = [
        _file(1, (64, 80), "JPEG", quality=50),
        _file(2, (72, 96, 3), "JPEG", quality=75, subsampling=2),
        _file(3, (48, 64, 3), "JPEG", quality=90, subsampling=0, progressive=True),
        _file(4, (40, 56, 3), "PNG"),
    ]
    options = ["--method", "tgv", "--iterations", "40", "--tolerance", "0"]
    alone = [native.decode(data, options) for data in files]
    together = [None] * len(files)
    errors = []

    def work(index: int) -> None:
        try:
            together[index] = native.decode(files[index], options)
        except BaseException as error:  # noqa: BLE001 -- raised below, on the main thread
            errors.append(error)

    threads = [threading.Thread(target=work, args=(index,)) for index in range(len(files))]
    for thread in threads:
        thread.start()
    for thread in threads:
        thread.join()
    assert not errors, errors
    for one, other in zip(alone, together):
        assert other is not None
        np.testing.assert_array_equal(one.picture.view(np.uint64), other.picture.view(np.uint64))
        np.testing.assert_array_equal(one.canvas.view(np.uint64), other.canvas.view(np.uint64))
