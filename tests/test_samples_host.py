"""The host model of pictures of rounded samples, without a GPU: each level's interval is the
closed interval of the doubles that round to it (docs/math.md 11; cpp/src/samples.cpp:86-105) --
the rational ends (v -+ 1/2) 255 / (2^b - 1) rounded inward, computed here again in exact
fractions -- the last level's upper end 255, the centre the double nearest to v s; with a slack,
the floating-point formula clipped to 0..255."""

import ctypes
import math
from fractions import Fraction

import numpy as np
import pytest

from oracle import output


def _interval(level: int, bits: int, slack: float = 0.0) -> tuple[float, float, float]:
    from unround import native

    library = native._library()
    library.unround_b200_sample_interval.restype = ctypes.c_int32
    library.unround_b200_sample_interval.argtypes = [ctypes.c_uint32, ctypes.c_int32, ctypes.c_double,
                                                     ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_size_t]
    ends = (ctypes.c_double * 3)()
    message = ctypes.create_string_buffer(256)
    status = library.unround_b200_sample_interval(level, bits, slack, ends, message, 256)
    assert status == 0, message.value
    return ends[0], ends[1], ends[2]


def _up(value: Fraction) -> float:
    """The least double at or above a non-negative rational."""
    near = float(value)
    return near if Fraction(near) >= value else math.nextafter(near, math.inf)


def _below(value: Fraction) -> float:
    """The greatest double below a positive rational."""
    near = float(value)
    return math.nextafter(near, 0.0) if Fraction(near) >= value else near


@pytest.mark.parametrize("bits", [1, 2, 4, 8, 10, 16])
def test_intervals_hold_the_values_that_round_to_their_level(bits):
    top = 2**bits - 1
    chosen = {0, 1, 2, top // 3, top // 2, top - 1, top} | set(np.random.default_rng(bits).integers(0, top + 1, 40).tolist())
    levels = sorted(v for v in chosen if 0 <= v <= top)
    for v in levels:
        lower, upper, centre = _interval(v, bits)
        assert lower == (0.0 if v == 0 else _up(Fraction(255 * (2 * v - 1), 2 * top)))
        assert upper == (255.0 if v == top else _below(Fraction(255 * (2 * v + 1), 2 * top)))
        assert centre == float(Fraction(255 * v, top))
        assert lower <= centre <= upper


def test_eight_bits_give_back_their_levels_when_rounded():
    for v in range(256):
        lower, upper, centre = _interval(v, 8)
        assert centre == v
        # Rounded halves away from 0 (exactly: floor(x + 1/2) in binary64 would lift
        # 0.49999999999999994), every value held rounds to v.
        assert output.rounded(lower, 1, 255) == v and output.rounded(upper, 1, 255) == v


def test_a_slack_widens_the_interval_within_0_and_255():
    lower, upper, _ = _interval(10, 8, slack=0.25)
    assert lower == (10 - 0.5 - 0.25) * 1.0 and upper == (10 + 0.5 + 0.25) * 1.0
    lower, upper, _ = _interval(0, 8, slack=1.0)
    assert lower == 0.0
    lower, upper, _ = _interval(255, 8, slack=1.0)
    assert upper == 255.0
