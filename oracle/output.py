"""Test infrastructure: the oracle of 8- and 16-bit output. A CPU restatement, in exact
rationals, of how the reference makes the levels of PNG and PNM files from binary64 samples
(docs/math.md 10 of JPEG-Unround; rust/unround/src/output.rs:66-209), in the form its own
tests state it (python/tests/test_native.py:552-629: `rounded`, `dithered`, the channels'
shifts of the matrix). Pinned by tests/test_output_oracle.py against those tests' own cases;
only tests use it, as the checker.

  rounded   output.rs:99-109    the exact product, rounded to the nearest, halves away from 0
  dithered  output.rs:77-89     floor of the exact product, or the level above where its
                                fraction reaches 1 - (2 rank + 1) / 8192
  levels    output.rs:134-185   sample c of pixel (i, j) at rank ((i + a) mod 64, (j + b) mod 64)
"""

from __future__ import annotations

import math
from fractions import Fraction

import numpy as np
import numpy.typing as npt

SHIFTS = {"apart": [(0, 0), (0, 32), (32, 0), (32, 32)], "together": [(0, 0)] * 4}


def rounded(value: float, scale: int, top: int) -> int:
    """value times scale, exactly, rounded to the nearest integer, halves away from 0, clamped."""
    exact = Fraction(value) * scale
    whole = int(abs(exact) + Fraction(1, 2)) * (1 if exact >= 0 else -1)
    return min(max(whole, 0), top)


def dithered(value: float, rank: int, scale: int, top: int) -> int:
    """The level of value times scale, exactly: its floor, or the level above where the fraction
    reaches 1 - (2 rank + 1) / 8192; clamped to 0 .. top."""
    y = Fraction(value) * scale
    whole = math.floor(y)
    above = y - whole >= 1 - Fraction(2 * rank + 1, 8192)
    return min(max(whole + int(above), 0), top)


def levels(picture: npt.ArrayLike, ranks: npt.NDArray, *, sixteen: bool, dither: str = "blue-noise",
           channels: str = "apart") -> npt.NDArray[np.int64]:
    """The levels (height, width, channels) of a small picture, sample by sample."""
    samples = np.asarray(picture, dtype=np.float64)
    stacked = samples.reshape(samples.shape[0], samples.shape[1], -1)
    scale, top = (257, 65535) if sixteen else (1, 255)
    out = np.zeros(stacked.shape, dtype=np.int64)
    for (row, column, channel), value in np.ndenumerate(stacked):
        if dither == "none":
            out[row, column, channel] = rounded(float(value), scale, top)
        else:
            down, across = SHIFTS[channels][channel]
            rank = int(ranks[(row + down) % 64, (column + across) % 64])
            out[row, column, channel] = dithered(float(value), rank, scale, top)
    return out
