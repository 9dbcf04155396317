"""The TIFF writer (unround_tiff; the reference's tests in python/tests/test_native.py:508-560, which
read files with tifffile, not in this image): the file read back here by a small reader of the
TIFF 6.0 specification -- the header, the first IFD's tags, the strip -- holds the picture's
binary64 samples bit for bit, uncompressed, SampleFormat IEEE, the samples per pixel, and declares
JFIF's YCbCr as the reference's does, an alpha as unassociated, and the ICC profile where it goes
with the picture. No GPU is needed."""

import struct

import numpy as np
import pytest

from unround import native

_TYPES = {1: ("B", 1), 2: ("c", 1), 3: ("H", 2), 4: ("I", 4), 5: ("II", 8), 7: ("B", 1), 16: ("Q", 8)}


def read_tiff(data: bytes) -> tuple[np.ndarray, dict[int, tuple]]:
    assert data[:4] == b"II*\x00"
    (offset,) = struct.unpack_from("<I", data, 4)
    (count,) = struct.unpack_from("<H", data, offset)
    tags = {}
    for e in range(count):
        tag, kind, n, value = struct.unpack_from("<HHII", data, offset + 2 + 12 * e)
        code, size = _TYPES[kind]
        where = offset + 2 + 12 * e + 8 if n * size <= 4 else value
        if kind == 5:
            tags[tag] = struct.unpack_from("<" + "I" * 2 * n, data, where)
        elif kind == 7:
            tags[tag] = (bytes(data[where : where + n]),)
        else:
            tags[tag] = struct.unpack_from("<" + code * n, data, where)
    assert struct.unpack_from("<I", data, offset + 2 + 12 * count)[0] == 0  # one IFD
    width, height, spp = tags[256][0], tags[257][0], tags[277][0]
    start, length = tags[273][0], tags[279][0]
    assert length == width * height * spp * 8
    samples = np.frombuffer(data, dtype="<f8", count=width * height * spp, offset=start)
    return samples.reshape((height, width, spp)), tags


def awkward(shape):
    samples = np.random.default_rng(60).uniform(-10.0, 265.0, size=shape)
    special = [-0.0, 0.0, 5e-324, -5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, 1.0 / 3.0, 255.0]
    flat = samples.reshape(-1)
    flat[: min(len(special), flat.size)] = special[: flat.size]
    return samples


@pytest.mark.parametrize("shape", [(1, 1), (7, 13), (21, 30), (5, 6, 3), (3, 5, 2), (4, 4, 4)])
def test_the_tiff_holds_the_samples_bit_for_bit(shape):
    picture = awkward(shape)
    read, tags = read_tiff(native.tiff_bytes(picture))
    spp = 1 if len(shape) == 2 else shape[2]
    assert tags[259] == (1,) and tags[258] == (64,) * spp and tags[339] == (3,) * spp and tags[284] == (1,)
    assert tags[262] == ((1,) if spp <= 2 else (2,))
    if spp in (2, 4):
        assert tags[338] == (2,)
    np.testing.assert_array_equal(read.reshape(picture.shape).view(np.uint64), picture.view(np.uint64))


def test_ycbcr_is_declared_as_it_is():
    planes = np.random.default_rng(3).uniform(0.0, 255.0, size=(6, 9, 3))
    read, tags = read_tiff(native.tiff_bytes(planes, ycbcr=True))
    assert tags[262] == (6,)
    assert tags[530] == (1, 1)
    assert tags[529] == (299, 1000, 587, 1000, 114, 1000)
    assert tags[532] == (0, 1, 255, 1, 128, 1, 255, 1, 128, 1, 255, 1)
    np.testing.assert_array_equal(read.view(np.uint64), planes.view(np.uint64))
    with pytest.raises(native.UnroundError):
        native.tiff_bytes(planes[:, :, 0], ycbcr=True)
    with pytest.raises(native.UnroundError):
        native.tiff_bytes(np.zeros((2, 2, 5)))
    with pytest.raises(ValueError, match="height, width"):
        native.tiff_bytes(np.zeros(4))


def _profile(space: bytes) -> bytes:
    header = bytearray(132)
    struct.pack_into(">I", header, 0, 132)
    header[8] = 4
    header[12:16] = b"mntr"
    header[16:20] = space
    header[20:24] = b"XYZ "
    header[36:40] = b"acsp"
    return bytes(header)


def test_icc_profiles():
    rgb, grey = _profile(b"RGB "), _profile(b"GRAY")
    picture = np.random.default_rng(4).uniform(0.0, 255.0, size=(4, 5, 3))
    assert read_tiff(native.tiff_bytes(picture, icc_profile=rgb))[1][34675] == (rgb,)
    assert read_tiff(native.tiff_bytes(picture, ycbcr=True, icc_profile=rgb))[1][34675] == (rgb,)
    assert read_tiff(native.tiff_bytes(picture[:, :, 0], icc_profile=grey))[1][34675] == (grey,)
    with pytest.warns(native.UnroundWarning, match="not written"):
        data = native.tiff_bytes(picture, icc_profile=grey)
    assert 34675 not in read_tiff(data)[1]
