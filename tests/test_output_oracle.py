"""The oracle of 8- and 16-bit output (oracle/output.py) pinned, without a GPU: its rounding on
the reference's own cases of halves (python/tests/test_native.py:569-591 of JPEG-Unround), its
dither keeping every level's mean over the matrix, and the library's blue-noise matrix against
the reference's (tests/golden/blue_noise_ranks.npy, from the reference's generator)."""

import ctypes
import math
from fractions import Fraction
from pathlib import Path

import numpy as np

from oracle import output

GOLDEN = Path(__file__).resolve().parent / "golden" / "blue_noise_ranks.npy"


def test_the_library_makes_the_reference_s_blue_noise_matrix():
    from unround import native

    library = native._library()
    library.unround_b200_blue_noise.restype = ctypes.c_int32
    library.unround_b200_blue_noise.argtypes = [ctypes.POINTER(ctypes.c_uint16), ctypes.c_char_p, ctypes.c_size_t]
    ranks = np.zeros(4096, dtype=np.uint16)
    message = ctypes.create_string_buffer(256)
    assert library.unround_b200_blue_noise(ranks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), message, 256) == 0
    golden = np.load(GOLDEN)
    np.testing.assert_array_equal(ranks.reshape(64, 64), golden)
    assert sorted(golden.ravel().tolist()) == list(range(4096))


def test_rounding_takes_halves_away_from_zero_and_clamps():
    cases = {0.5: 1, 1.5: 2, 2.5: 3, 254.5: 255, 0.49999999999999994: 0, -0.5: 0, 255.4: 255, 255.5: 255,
             300.0: 255, -7.0: 0, 128.0: 128}
    for value, level in cases.items():
        assert output.rounded(value, 1, 255) == level, value
    assert output.rounded(128.0, 257, 65535) == 32896
    assert output.rounded(255.0, 257, 65535) == 65535


def test_sixteen_bits_round_the_exact_product():
    # Samples whose product with 257 rounds (in binary64) onto a half from below: the exact
    # product is below the half, so the level is its floor.
    found = 0
    for whole in range(16, 400):
        target = whole + 0.5
        near = target / 257
        for sample in (math.nextafter(near, 0.0), near, math.nextafter(near, 256.0)):
            if sample * 257 == target and Fraction(sample) * 257 < Fraction(target):
                assert output.rounded(sample, 257, 65535) == math.floor(sample * 257)
                found += 1
    assert found > 100


def test_over_the_matrix_a_level_keeps_its_mean():
    ranks = np.load(GOLDEN)
    for value in (0.0, 7.25, 100.0 + 1 / 4096, 200.0 + 4095 / 4096, 128.5):
        mean = Fraction(sum(output.dithered(value, int(r), 1, 255) for r in ranks.ravel()), 4096)
        assert mean == Fraction(value), value


def test_levels_take_the_matrix_shifted_apart_or_alike():
    ranks = np.load(GOLDEN)
    picture = np.full((3, 4, 3), 9.5)
    apart = output.levels(picture, ranks, sixteen=False, channels="apart")
    together = output.levels(picture, ranks, sixteen=False, channels="together")
    assert (together[..., 0] == together[..., 1]).all() and (together[..., 1] == together[..., 2]).all()
    for channel, (down, across) in enumerate(output.SHIFTS["apart"][:3]):
        expected = [[9 + int(Fraction(1, 2) >= 1 - Fraction(2 * int(ranks[(i + down) % 64, (j + across) % 64]) + 1,
                                                                8192)) for j in range(4)] for i in range(3)]
        np.testing.assert_array_equal(apart[..., channel], expected)
