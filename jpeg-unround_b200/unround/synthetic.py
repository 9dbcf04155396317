"""Seeded synthetic pictures and their JPEG levels, standing in for the reference's image sets.

The reference benchmarks on its own synthetic set and on photographs (scripts/test_images.py,
scripts/fetch_datasets.py of JPEG-Unround), which are not here; its tests quantize pictures in
memory without entropy coding (rust/unround/tests/support/synthetic.rs). This module does the
same from a seed: a piecewise-smooth picture -- random axis-aligned rectangles with linear
ramps and Gaussian blobs over a ramp, clipped to 0..255 and rounded to 8 bits -- optionally
with Gaussian noise, quantized by the orthonormal 8x8 DCT of the level-shifted samples with a
quality-scaled standard table (ITU-T T.81 Annex K, IJG scaling), levels rounded half to even.
Colour pictures go through JFIF's YCbCr and 2x2 (or other) chroma means, as an encoder does.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import numpy.typing as npt

from unround import jpegio

# T.81 Annex K, Tables K.1 and K.2, in natural order.
LUMA = np.array(
    [16, 11, 10, 16, 24, 40, 51, 61, 12, 12, 14, 19, 26, 58, 60, 55, 14, 13, 16, 24, 40, 57, 69, 56,
     14, 17, 22, 29, 51, 87, 80, 62, 18, 22, 37, 56, 68, 109, 103, 77, 24, 35, 55, 64, 81, 104, 113, 92,
     49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99], dtype=np.int64)
CHROMA = np.array(
    [17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99, 24, 26, 56, 99, 99, 99, 99, 99,
     47, 66, 99, 99, 99, 99, 99, 99] + [99] * 32, dtype=np.int64)


def table(base: npt.NDArray[np.int64], quality: int) -> npt.NDArray[np.uint16]:
    """The IJG scaling of a base table to a quality 1..100, entries 1..255 (baseline)."""
    quality = min(max(int(quality), 1), 100)
    scale = 5000 // quality if quality < 50 else 200 - 2 * quality
    return np.clip((base * scale + 50) // 100, 1, 255).astype(np.uint16)


def _basis() -> npt.NDArray[np.float64]:
    k = np.arange(8)[:, None]
    n = np.arange(8)[None, :]
    c = np.cos(np.pi * (2 * n + 1) * k / 16) * 0.5
    c[0, :] = np.sqrt(1 / 8)
    return c


BASIS = _basis()


def picture(rows: int, columns: int, rng: np.random.Generator, *, rectangles: int = 12, blobs: int = 20,
            sigma: tuple[float, float] = (5.0, 60.0), amplitude: float = 60.0, noise: float = 0.0) -> npt.NDArray[np.float64]:
    """A piecewise-smooth picture of 8-bit samples (as float64)."""
    y = np.arange(rows, dtype=np.float64)[:, None]
    x = np.arange(columns, dtype=np.float64)[None, :]
    base = rng.uniform(60, 190)
    out = base + rng.uniform(-40, 40) * (y / rows) + rng.uniform(-40, 40) * (x / columns)
    out = np.broadcast_to(out, (rows, columns)).copy()
    for _ in range(rectangles):
        y0, y1 = np.sort(rng.integers(0, rows, 2))
        x0, x1 = np.sort(rng.integers(0, columns, 2))
        y1, x1 = max(y1, y0 + 1), max(x1, x0 + 1)
        level = rng.uniform(20, 235)
        gy = rng.uniform(-60, 60) / max(y1 - y0, 1)
        gx = rng.uniform(-60, 60) / max(x1 - x0, 1)
        out[y0:y1, x0:x1] = level + gy * (y[y0:y1] - y0) + gx * (x[:, x0:x1] - x0)
    for _ in range(blobs):
        cy, cx = rng.uniform(0, rows), rng.uniform(0, columns)
        s = rng.uniform(*sigma)
        a = rng.uniform(-amplitude, amplitude)
        ya, yb = max(int(cy - 3 * s), 0), min(int(cy + 3 * s) + 1, rows)
        xa, xb = max(int(cx - 3 * s), 0), min(int(cx + 3 * s) + 1, columns)
        if ya >= yb or xa >= xb:
            continue
        d2 = (y[ya:yb] - cy) ** 2 + (x[:, xa:xb] - cx) ** 2
        out[ya:yb, xa:xb] += a * np.exp(-d2 / (2 * s * s))
    if noise > 0:
        out += rng.normal(0.0, noise, size=out.shape)
    return np.rint(np.clip(out, 0, 255))


def pad(samples: npt.NDArray[np.float64], rows: int, columns: int) -> npt.NDArray[np.float64]:
    """The samples extended to rows x columns by repeating the last row and column."""
    return np.pad(samples, ((0, rows - samples.shape[0]), (0, columns - samples.shape[1])), mode="edge")


def quantize(samples: npt.NDArray[np.float64], steps: npt.NDArray[np.uint16]) -> npt.NDArray[np.int16]:
    """The levels (rows/8, columns/8, 8, 8) of samples whose sides are multiples of 8:
    round-half-even of DCT(samples - 128) / Q."""
    rows, columns = samples.shape
    blocks = (samples - 128.0).reshape(rows // 8, 8, columns // 8, 8).transpose(0, 2, 1, 3)
    coefficients = np.einsum("kn,abnm,lm->abkl", BASIS, blocks, BASIS, optimize=True)
    q = steps.reshape(8, 8).astype(np.float64)
    return np.rint(coefficients / q).astype(np.int16)


def dequantize(levels: npt.NDArray[np.int16], steps: npt.NDArray[np.uint16]) -> npt.NDArray[np.float64]:
    """The standard decoder's samples (the inverse DCT of q Q, + 128), unclamped."""
    coefficients = levels.astype(np.float64) * steps.reshape(8, 8).astype(np.float64)
    blocks = np.einsum("kn,abkl,lm->abnm", BASIS, coefficients, BASIS, optimize=True)
    a, b = levels.shape[:2]
    return blocks.transpose(0, 2, 1, 3).reshape(a * 8, b * 8) + 128.0


@dataclass(frozen=True)
class Synthetic:
    """A synthetic picture: its samples (H, W) or (H, W, 3), and its quantized image."""

    samples: npt.NDArray[np.float64]
    image: jpegio.Image


def grey(rows: int, columns: int, *, quality: int = 50, seed: int = 0, noise: float = 0.0,
         steps: npt.ArrayLike | None = None) -> Synthetic:
    """A greyscale picture and its levels: the standard luminance table at the quality, or the
    steps given (64, natural order)."""
    rng = np.random.default_rng(seed)
    samples = picture(rows, columns, rng, noise=noise)
    q = table(LUMA, quality) if steps is None else np.asarray(steps, dtype=np.uint16).reshape(64)
    padded = pad(samples, -(-rows // 8) * 8, -(-columns // 8) * 8)
    levels = quantize(padded, q)
    return Synthetic(samples, jpegio.image_of(rows, columns, jpegio.ColorSpace.GRAYSCALE, [(levels, q, 1, 1)]))


# JFIF's YCbCr (ITU-T T.871), in binary64.
def ycbcr(rgb: npt.NDArray[np.float64]) -> npt.NDArray[np.float64]:
    r, g, b = rgb[..., 0], rgb[..., 1], rgb[..., 2]
    y = 0.299 * r + 0.587 * g + 0.114 * b
    return np.stack([y, 128 + (b - y) / 1.772, 128 + (r - y) / 1.402])


def colour(rows: int, columns: int, *, quality: int = 75, seed: int = 0, noise: float = 0.0,
           sampling: tuple[int, int] = (2, 2)) -> Synthetic:
    """A colour picture (the generator per RGB channel) and its YCbCr levels with chroma cells of
    sampling = (down, across) luma samples: (2, 2) is 4:2:0, (1, 2) 4:2:2, (1, 1) 4:4:4."""
    rng = np.random.default_rng(seed)
    rgb = np.stack([picture(rows, columns, rng, noise=noise) for _ in range(3)], axis=-1)
    planes = np.clip(np.rint(ycbcr(rgb)), 0, 255)
    down, across = sampling
    mcu_rows, mcu_columns = 8 * down, 8 * across
    height, width = -(-rows // mcu_rows) * mcu_rows, -(-columns // mcu_columns) * mcu_columns
    luma_q, chroma_q = table(LUMA, quality), table(CHROMA, quality)
    components = []
    y = pad(planes[0], height, width)
    y_rows, y_columns = -(-rows // 8), -(-columns // 8)
    components.append((quantize(y, luma_q)[:y_rows, :y_columns], luma_q, across, down))
    for plane in planes[1:]:
        padded = pad(plane, height, width)
        means = np.rint(padded.reshape(height // down, down, width // across, across).mean(axis=(1, 3)))
        c_rows, c_columns = -(-rows // mcu_rows), -(-columns // mcu_columns)
        c = pad(means, -(-means.shape[0] // 8) * 8, -(-means.shape[1] // 8) * 8)
        components.append((quantize(c, chroma_q)[:c_rows, :c_columns], chroma_q, 1, 1))
    return Synthetic(rgb, jpegio.image_of(rows, columns, jpegio.ColorSpace.YCBCR, components))


def large(side: int = 8192, *, seed: int = 5) -> Synthetic:
    """A large greyscale picture (the generator plus Gaussian noise sigma 2) quantized with a
    custom table of steps drawn uniformly from 1..64 (a custom table: no quality factor applies)."""
    steps = np.random.default_rng(seed).integers(1, 65, size=64)
    return grey(side, side, seed=seed, noise=2.0, steps=steps)


@dataclass(frozen=True)
class MixEntry:
    """A picture of a mix and the options it is solved with."""

    image: jpegio.Image
    options: list[str]
    colour: bool
    method: str
    quality: int
    alpha: float


def mix(count: int = 64, *, seed: int = 3, smallest: int = 256, largest: int = 2048, iterations: int = 300,
        noise: float = 2.0) -> list[MixEntry]:
    """A seeded mix of pictures of uneven sizes and settings, as a batch of many users' requests:
    sides drawn uniformly from the multiples of 16 in [smallest, largest], greyscale or 4:2:0
    colour with equal odds, quality uniform in 10..90, TV or TGV with equal odds, alpha
    log-uniform in [0.3, 3] (TGV: alpha1 = alpha, alpha0 = 2 alpha), `iterations` iterations, no
    tolerance, a record at the last iteration only."""
    rng = np.random.default_rng(seed)
    sides = np.arange(smallest, largest + 1, 16)
    out = []
    for n in range(count):
        rows, columns = int(rng.choice(sides)), int(rng.choice(sides))
        colour_picture = bool(rng.integers(0, 2))
        quality = int(rng.integers(10, 91))
        tgv = bool(rng.integers(0, 2))
        alpha = float(np.exp(rng.uniform(np.log(0.3), np.log(3.0))))
        picture_seed = int(rng.integers(0, 2**31))
        made = (colour(rows, columns, quality=quality, seed=picture_seed, noise=noise) if colour_picture
                else grey(rows, columns, quality=quality, seed=picture_seed, noise=noise))
        common = ["--iterations", str(iterations), "--tolerance", "0", "--record-every", "0"]
        if tgv:
            options = ["--method", "tgv", "--alpha1", repr(alpha), "--alpha0", repr(2 * alpha), *common]
        else:
            options = ["--method", "tv", "--alpha", repr(alpha), *common]
        out.append(MixEntry(made.image, options, colour_picture, "tgv" if tgv else "tv", quality, alpha))
    return out
