"""Test infrastructure: the oracle. A CPU restatement, in NumPy, of the reference's TV/TGV
primal-dual reconstruction (docs/math.md of JPEG-Unround), whole-canvas array operations in
the natural layout.

Pinned against the reference's golden vectors (tests/golden, from conformance/cases) and
against the reference's own C++ solver (oracle/_ref) by the tests. Only tests and the bench's
CPU-baseline leg use it, as the checker; nothing of the product imports it.

It computes in the dtype given (float64 by default): run in float32 it restates the binary32
arithmetic of the device iterations operation for operation, which isolates the rounding of
binary32 from the device code.

Functions cite the reference (file:line) whose computation they restate:
  dct / idct          cpp/src/dct.cpp:246-278 (columns then rows; rows then columns)
  Component           cpp/src/model.cpp:134-256 (intervals, weights, flat blocks, centres)
  laplace_*           cpp/src/laplace.cpp:81-146
  plan                cpp/src/pdhg.cpp:147-233
  prox / conjugate    cpp/src/model.cpp:57-111, cpp/src/frames.cpp:302-360, 428-487
  iterate             cpp/src/primal_dual.hpp:525-735
  record              cpp/src/primal_dual.hpp:446-501, 836-895
  solve               cpp/src/primal_dual.hpp:957-1013
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

# cos(pi j / 16), j = 0..8, the doubles nearest to the exact values (docs/math.md 1.1).
_COS = [float.fromhex(h) for h in ("0x1p0", "0x1.f6297cff75cb0p-1", "0x1.d906bcf328d46p-1", "0x1.a9b66290ea1a3p-1",
                                    "0x1.6a09e667f3bcdp-1", "0x1.1c73b39ae68c8p-1", "0x1.87de2a6aea963p-2",
                                    "0x1.8f8b83c69a60bp-3", "0x0p0")]
_ROOT_EIGHTH = float.fromhex("0x1.6a09e667f3bcdp-2")


def _cosine(m: int) -> float:
    if m <= 8:
        return _COS[m]
    if m <= 16:
        return -_COS[16 - m]
    if m <= 24:
        return -_COS[m - 16]
    return _COS[32 - m]


BASIS = np.array([[_ROOT_EIGHTH if k == 0 else 0.5 * _cosine(((2 * n + 1) * k) % 32) for n in range(8)]
                  for k in range(8)])


def dct(blocks: np.ndarray) -> np.ndarray:
    """D of 8x8 blocks (..., 8, 8) [m, n] -> [v, u]: down the columns, then along the rows."""
    c = BASIS.astype(blocks.dtype)
    return np.matmul(np.matmul(c, blocks), c.T)


def idct(coefficients: np.ndarray) -> np.ndarray:
    """D^T: along the rows, then down the columns."""
    c = BASIS.astype(coefficients.dtype)
    return np.matmul(c.T, np.matmul(coefficients, c))


def _blocks(grid: np.ndarray, rows: int, columns: int) -> np.ndarray:
    return grid[: 8 * rows, : 8 * columns].reshape(rows, 8, columns, 8).transpose(0, 2, 1, 3)


def _grid(blocks: np.ndarray) -> np.ndarray:
    rows, columns = blocks.shape[:2]
    return blocks.transpose(0, 2, 1, 3).reshape(8 * rows, 8 * columns)


# --- Finite differences (docs/math.md 3; cpp/src/operators.cpp:46-150) -------------------------

def dx_forward(f: np.ndarray) -> np.ndarray:
    out = np.zeros_like(f)
    out[:, :-1] = f[:, 1:] - f[:, :-1]
    return out


def dy_forward(f: np.ndarray) -> np.ndarray:
    out = np.zeros_like(f)
    out[:-1, :] = f[1:, :] - f[:-1, :]
    return out


def dx_backward(f: np.ndarray) -> np.ndarray:
    """f[i, j] (not in the last column) - f[i, j - 1] (not in the first)."""
    if f.shape[1] == 1:
        return np.zeros_like(f)
    own = f.copy()
    own[:, -1] = 0
    before = np.zeros_like(f)
    before[:, 1:] = f[:, :-1]
    return own - before


def dy_backward(f: np.ndarray) -> np.ndarray:
    if f.shape[0] == 1:
        return np.zeros_like(f)
    own = f.copy()
    own[-1, :] = 0
    before = np.zeros_like(f)
    before[1:, :] = f[:-1, :]
    return own - before


def divergence(p1: np.ndarray, p2: np.ndarray) -> np.ndarray:
    return dy_backward(p2) + dx_backward(p1)


def sym_gradient(w1: np.ndarray, w2: np.ndarray):
    half = np.asarray(0.5, dtype=w1.dtype)
    return dx_backward(w1), dy_backward(w2), half * (dy_backward(w1) + dx_backward(w2))


def div2(r11, r22, r12):
    return dx_forward(r11) + dy_forward(r12), dx_forward(r12) + dy_forward(r22)


def ball_scale(square: np.ndarray, radius: float) -> np.ndarray:
    norm = np.sqrt(square)
    radius = np.asarray(radius, dtype=square.dtype)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(norm > radius, radius / norm, np.asarray(1, dtype=square.dtype))


# --- The model (docs/math.md 1.2, 2, 4.1; cpp/src/model.cpp, cpp/src/laplace.cpp) ----------------

_SERIES = [float(Fraction(b) / math.factorial(2 * k)) for k, b in enumerate(
    [Fraction(1, 6), Fraction(-1, 30), Fraction(1, 42), Fraction(-1, 30), Fraction(5, 66), Fraction(-691, 2730),
     Fraction(7, 6), Fraction(-3617, 510), Fraction(43867, 798), Fraction(-174611, 330), Fraction(854513, 138)], 1)]


def laplace_scale(zeros: int, others: int, total: int, step: float) -> float:
    """cpp/src/laplace.cpp:81-107: the maximum-likelihood Laplace scale."""
    if total == 0:
        return 0.0
    a = zeros + total + 2 * others
    discriminant = zeros * zeros + 4 * a * total
    root = math.sqrt(float(discriminant))
    t = float(2 * total) / (float(zeros) + root)
    if t >= 0.5:
        top = float(8 * total * (zeros + others))
        first = root + float(2 * total - zeros)
        second = float(zeros) + root
        log_inverse = -math.log1p(-(top / (first * second)))
    else:
        log_inverse = -math.log(t)
    return step / (2.0 * log_inverse)


def laplace_shrinkage(rho: float) -> float:
    """cpp/src/laplace.cpp:132-146: delta / Q of a bin's mean."""
    if not rho > 0:
        return 0.0
    if math.isinf(rho):
        return 0.5
    if rho < 1.0:
        square = rho * rho
        total = _SERIES[10]
        for k in range(9, -1, -1):
            total = total * square + _SERIES[k]
        return total * rho
    return (0.5 - 1.0 / rho) + math.exp(-rho) / -math.expm1(-rho)


@dataclass
class DataTerm:
    """The options of G (cpp/include/unround/model.hpp:41-66)."""

    mu: float | None = None
    mu_scale: float = 9.0
    mu_power: float = 0.9
    mu_chroma: float = 0.3
    slack: float = 0.0
    dc_weight: float = 1.0
    centres: str = "midpoint"
    power: float = 2.0
    slack_cost: float = 0.0
    flat_weight: float = 0.1
    flat_levels: int = 0
    flat_dc: int | None = 1


@dataclass
class Component:
    """One component's problem (cpp/src/model.cpp:134-256)."""

    levels: np.ndarray  # (rows, columns, 8, 8) int16
    steps: np.ndarray   # (8, 8)
    weights: np.ndarray
    flat_weights: np.ndarray
    flat: np.ndarray    # (rows, columns) bool
    lower: np.ndarray
    upper: np.ndarray
    centres: np.ndarray
    inner_lower: np.ndarray | None
    inner_upper: np.ndarray | None
    costs: np.ndarray | None
    cells: tuple[int, int] = (1, 1)


def make_component(levels: np.ndarray, table: np.ndarray, data: DataTerm, cells=(1, 1)) -> Component:
    levels = np.asarray(levels, dtype=np.int16)
    steps = np.asarray(table, dtype=np.float64).reshape(8, 8)
    if data.mu is not None:
        mu = data.mu
    else:
        mean = float(int(np.sum(np.asarray(table, dtype=np.int64)))) / 64.0
        mu = data.mu_scale * mean if data.mu_power == 1.0 else data.mu_scale * math.pow(mean, data.mu_power)
    if data.power == 2.0:
        powered = steps * steps
    elif data.power == 1.0:
        powered = steps
    else:
        powered = np.power(steps, data.power)
    weights = mu / powered
    weights[0, 0] *= data.dc_weight
    flat_weights = weights * data.flat_weight
    q = levels.astype(np.float64)
    nonzero = np.count_nonzero(levels.reshape(*levels.shape[:2], 64)[..., 1:], axis=-1)
    flat = nonzero <= data.flat_levels
    if data.flat_dc is not None:
        dc = levels[..., 0, 0].astype(np.int64)
        near = np.ones_like(flat)
        bound = data.flat_dc
        near[1:, :] &= np.abs(dc[1:, :] - dc[:-1, :]) <= bound
        near[:-1, :] &= np.abs(dc[:-1, :] - dc[1:, :]) <= bound
        near[:, 1:] &= np.abs(dc[:, 1:] - dc[:, :-1]) <= bound
        near[:, :-1] &= np.abs(dc[:, :-1] - dc[:, 1:]) <= bound
        flat &= near
    shift = np.zeros((8, 8))
    shift[0, 0] = 1024.0
    lower = ((q - 0.5) - data.slack) * steps + shift
    upper = ((q + 0.5) + data.slack) * steps + shift
    centres = q * steps + shift
    if data.centres == "mmse":
        flat_levels = levels.reshape(-1, 64).astype(np.int64)
        shrink = np.zeros(64)
        for k in range(1, 64):
            column = flat_levels[:, k]
            zeros = int(np.sum(column == 0))
            others = int(column.size - zeros)
            total = int(np.sum(np.where(column != 0, 2 * np.abs(column) - 1, 0)))
            scale = laplace_scale(zeros, others, total, float(steps.ravel()[k]))
            rho = float(steps.ravel()[k]) / scale if scale > 0 else math.inf
            shrink[k] = laplace_shrinkage(rho)
        shrink = shrink.reshape(8, 8)
        size = (np.abs(q) - shrink) * steps
        mmse = np.where(q == 0, 0.0, np.where(q < 0, -size, size))
        mmse[..., 0, 0] = centres[..., 0, 0]
        centres = mmse
    inner_lower = inner_upper = costs = None
    if data.slack > 0 and data.slack_cost > 0:
        inner_lower = (q - 0.5) * steps + shift
        inner_upper = (q + 0.5) * steps + shift
        costs = data.slack_cost / steps
    return Component(levels, steps, weights, flat_weights, flat, lower, upper, centres, inner_lower, inner_upper,
                     costs, cells)


def _weights_of(component: Component) -> np.ndarray:
    """Each coefficient's weight m (rows, columns, 8, 8): flat blocks take the flat weights."""
    return np.where(component.flat[..., None, None], component.flat_weights, component.weights)


def prox_coefficients(e: np.ndarray, step: float, component: Component, dtype) -> np.ndarray:
    """cpp/src/model.cpp:57-72, 483-539: zeta = clip((e + t c) r), with a slack's cost."""
    m = _weights_of(component)
    t = (step * m).astype(dtype)
    r = (1.0 / (1.0 + step * m)).astype(dtype)
    centre = component.centres.astype(dtype)
    low, high = component.lower.astype(dtype), component.upper.astype(dtype)
    z = (e + t * centre) * r
    if component.costs is None:
        return np.minimum(np.maximum(z, low), high)
    h = (step * component.costs * (1.0 / (1.0 + step * m))).astype(dtype)
    own_low, own_high = component.inner_lower.astype(dtype), component.inner_upper.astype(dtype)
    above = np.maximum(own_high, z - h)
    below = np.minimum(own_low, z + h)
    inside = np.where(z < own_low, below, z)
    return np.minimum(np.maximum(np.where(z > own_high, above, inside), low), high)


def conjugate_terms(s: np.ndarray, component: Component) -> np.ndarray:
    """cpp/src/model.cpp:74-111: g*(s) of each coefficient."""
    m = _weights_of(component)
    centre, low, high = component.centres, component.lower, component.upper
    with np.errstate(divide="ignore", invalid="ignore"):
        if component.costs is None:
            best = np.minimum(np.maximum(centre + s / m, low), high)
            away = best - centre
            weighted = s * best - 0.5 * m * (away * away)
            support = np.maximum(s * low, s * high)
            return np.where(m > 0, weighted, support)
        lam = component.costs
        own_low, own_high = component.inner_lower, component.inner_upper
        free = centre + s / m
        upward = np.minimum(np.maximum(centre + (s - lam) / m, own_high), high)
        downward = np.minimum(np.maximum(centre + (s + lam) / m, low), own_low)
        within = np.where(free < own_low, downward, free)
        weighted = np.where(free > own_high, upward, within)
        flat_best = np.where(s > 0, np.where(s > lam, high, own_high), np.where(s < -lam, low, own_low))
        best = np.where(m > 0, weighted, flat_best)
        away = best - centre
        beyond = np.maximum(np.maximum(best - own_high, own_low - best), 0.0)
        return s * best - 0.5 * m * (away * away) - lam * beyond


def value_terms(c: np.ndarray, component: Component) -> np.ndarray:
    m = _weights_of(component)
    away = c - component.centres
    out = 0.5 * m * (away * away)
    if component.costs is not None:
        out = out + component.costs * np.maximum(
            np.maximum(c - component.inner_upper, component.inner_lower - c), 0.0)
    return out


# --- The frame (docs/math.md 1.3, 4.4; cpp/src/frames.cpp) -------------------------------------

@dataclass
class Frame:
    height: int
    width: int
    rows: int
    columns: int
    components: list[Component]
    color_space: int = 1

    def free(self, c: int) -> bool:
        comp = self.components[c]
        down, across = comp.cells
        rows, columns = comp.levels.shape[:2]
        return down * across > 1 or 8 * rows * down < self.rows or 8 * columns * across < self.columns


def make_frame(height: int, width: int, color_space: int, components, data: list[DataTerm]) -> Frame:
    """cpp/src/frames.cpp:155-231: components = [(levels, table, h, v)]."""
    count = len(components)
    if count == 1:
        levels, table, _, _ = components[0]
        comp = make_component(levels, table, data[0])
        rows, columns = 8 * comp.levels.shape[0], 8 * comp.levels.shape[1]
        return Frame(height, width, rows, columns, [comp], color_space)
    h_max = max(h for _, _, h, _ in components)
    v_max = max(v for _, _, _, v in components)
    made = []
    for index, (levels, table, h, v) in enumerate(components):
        down, across = v_max // v, h_max // h
        term = data[0] if len(data) == 1 else data[index]
        if color_space == 2 and index > 0 and term.mu is None:
            term = DataTerm(**{**term.__dict__, "mu_scale": term.mu_scale * term.mu_chroma})
        made.append(make_component(levels, table, term, (down, across)))
    rows = 8 * v_max * -(-height // (8 * v_max))
    columns = 8 * h_max * -(-width // (8 * h_max))
    return Frame(height, width, rows, columns, made, color_space)


def _cell_sums(x: np.ndarray, component: Component) -> np.ndarray:
    down, across = component.cells
    rows, columns = component.levels.shape[:2]
    part = x[: 8 * rows * down, : 8 * columns * across]
    sums = part.reshape(8 * rows, down, 8 * columns * across).sum(axis=1)
    return sums.reshape(8 * rows, 8 * columns, across).sum(axis=2)


def prox_channel(v: np.ndarray, tau: float, component: Component, dtype) -> tuple[np.ndarray, np.ndarray]:
    """cpp/src/frames.cpp:302-360: x~ = v + spread(D^T zeta - mean v), zeta the prox at step
    tau / n_c of the DCT of the cell means; D^T zeta on the blocks where cells have one sample."""
    down, across = component.cells
    cells = down * across
    rows, columns = component.levels.shape[:2]
    if cells == 1:
        means = v[: 8 * rows, : 8 * columns]
    else:
        means = (_cell_sums(v, component) / np.asarray(cells, dtype=dtype)).astype(dtype)
    if np.dtype(dtype) == np.float64:
        e = dct(_blocks(means, rows, columns))
        zeta = prox_coefficients(e, tau / cells, component, dtype)
        back = _grid(idct(zeta))
        change_of = back - means
    else:
        # The device's binary32 arithmetic: each block centred on the middle of its DC interval
        # over 8 (exact in binary32), DC clipped on the centred interval; the same map in exact
        # arithmetic.
        middle_dc = component.levels[..., 0, 0].astype(np.float64) * component.steps[0, 0] + 1024.0
        middle = np.repeat(np.repeat((middle_dc / 8.0).astype(dtype), 8, axis=0), 8, axis=1)
        centred = means - middle
        e = dct(_blocks(centred, rows, columns))
        shifted = Component(**{**component.__dict__})
        shift = np.zeros_like(component.lower)
        shift[..., 0, 0] = middle_dc
        shifted.lower, shifted.upper, shifted.centres = component.lower - shift, component.upper - shift, component.centres - shift
        if component.costs is not None:
            shifted.inner_lower, shifted.inner_upper = component.inner_lower - shift, component.inner_upper - shift
        zeta_centred = prox_coefficients(e, tau / cells, shifted, dtype)
        zeta = zeta_centred.astype(np.float64) + shift
        inverse = _grid(idct(zeta_centred))
        back = inverse + middle
        change_of = inverse - centred
    out = v.copy()
    if cells == 1:
        out[: 8 * rows, : 8 * columns] = back
    else:
        change = np.repeat(np.repeat(change_of, down, axis=0), across, axis=1)
        out[: 8 * rows * down, : 8 * columns * across] += change
    return out, zeta


def start_canvas(frame: Frame, c: int, coefficients: np.ndarray, beyond: float = 128.0) -> np.ndarray:
    """cpp/src/frames.cpp:373-405: the inverse DCT spread over the cells, `beyond` past the blocks."""
    comp = frame.components[c]
    down, across = comp.cells
    samples = _grid(idct(coefficients))
    out = np.full((frame.rows, frame.columns), beyond)
    spread = np.repeat(np.repeat(samples, down, axis=0), across, axis=1)
    out[: spread.shape[0], : spread.shape[1]] = spread
    return out


def conjugate(frame: Frame, c: int, xi: np.ndarray, radius: float) -> float:
    """cpp/src/frames.cpp:428-493: g*(A xi / nu) plus the free samples' box terms."""
    comp = frame.components[c]
    rows, columns = comp.levels.shape[:2]
    down, across = comp.cells
    if down * across == 1:
        sums = xi[: 8 * rows, : 8 * columns]
    else:
        sums = _cell_sums(xi, comp)
    s = dct(_blocks(sums, rows, columns))
    total = float(np.sum(conjugate_terms(s, comp)))
    if frame.free(c):
        means = sums / (down * across)
        spread = np.repeat(np.repeat(means, down, axis=0), across, axis=1)
        inside = np.zeros_like(xi, dtype=bool)
        inside[: spread.shape[0], : spread.shape[1]] = True
        full = np.zeros_like(xi)
        full[: spread.shape[0], : spread.shape[1]] = spread
        terms = np.where(inside, radius * np.abs(xi - full), 128.0 * xi + radius * np.abs(xi))
        total += float(np.sum(terms))
    return total


# --- The method (docs/math.md 5, 6; cpp/src/pdhg.cpp, cpp/src/primal_dual.hpp) ------------------

@dataclass
class Plan:
    tgv: bool
    tau: float
    sigma: float
    iterations: int
    tolerance: float = 0.0
    relative_tolerance: float = 0.0
    partial_tolerance: float = 0.0
    partial_radius: float | None = None
    relaxation: float = 1.9
    record_every: int = 10
    free_radius: float = 255.0
    weights: list[float] = field(default_factory=lambda: [1.0])
    coupled: bool = True
    alpha: float = 1.0
    alpha1: float = 1.0
    alpha0: float = 2.0


def plan(tgv: bool, channels: int, *, alpha=1.0, alpha1=1.0, alpha0=2.0, iterations=None, tolerance=None,
         step_ratio=None, step_product=0.99, norm_squared=None, relaxation=1.9, record_every=10,
         weight_scaling=True, channel_weights=None, coupled=True, partial_radius=None, free_radius=255.0,
         relative_tolerance=0.0, partial_tolerance=0.0) -> Plan:
    """cpp/src/pdhg.cpp:147-233."""
    weights = list(channel_weights) if channel_weights else [1.0] * channels
    largest = max(weights)
    bound = (17.0 + math.sqrt(33.0)) / 2.0 if tgv else 8.0
    l2 = norm_squared if norm_squared is not None else bound * (largest * largest)
    weight = alpha1 if tgv else alpha
    default_ratio, default_tolerance = (3.0, 2e-3) if tgv else (10.0, 2e-4)
    ratio = step_ratio if step_ratio is not None else (default_ratio / (weight * weight) if weight_scaling else default_ratio)
    tol = tolerance if tolerance is not None else (default_tolerance * weight if weight_scaling else default_tolerance)
    most = iterations if iterations is not None else (10000 if tgv else 5000)
    return Plan(tgv, math.sqrt((ratio * step_product) / l2), math.sqrt(step_product / (ratio * l2)), most, tol,
                relative_tolerance, partial_tolerance, partial_radius, relaxation, record_every, free_radius,
                weights, coupled and channels > 1, alpha, alpha1, alpha0)


@dataclass
class State:
    x: list[np.ndarray]
    p: list[tuple[np.ndarray, np.ndarray]]
    w: list[tuple[np.ndarray, np.ndarray]]
    r: list[tuple[np.ndarray, np.ndarray, np.ndarray]]


def _project(fields: list[tuple[np.ndarray, ...]], radius: float, coupled: bool, tensor: bool) -> list[tuple]:
    def square(f):
        return f[0] * f[0] + f[1] * f[1] + (2 * (f[2] * f[2]) if tensor else 0)

    if coupled:
        total = sum(square(f) for f in fields)
        scale = ball_scale(total, radius)
        return [tuple(a * scale for a in f) for f in fields]
    return [tuple(a * ball_scale(square(f), radius) for a in f) for f in fields]


@dataclass
class Solved:
    canvas: np.ndarray
    coefficients: list[np.ndarray]
    records: list[tuple[int, float, float, float, float]]
    iterations: int
    stop: int


def solve(frame: Frame, p: Plan, *, dtype=np.float64, start: dict | None = None, observer=None) -> Solved:
    """cpp/src/primal_dual.hpp:957-1013: records at 0 (unless only the last is), every
    record_every iterations and at the last; stop at the first record that meets a tolerance."""
    dt = np.dtype(dtype)
    C = len(frame.components)
    zero = lambda: np.zeros((frame.rows, frame.columns), dtype=dt)  # noqa: E731
    xs, zetas = [], []
    offset = 0
    for c, comp in enumerate(frame.components):
        if start is not None and start.get("coefficients") is not None:
            count = comp.levels.size
            given = np.asarray(start["coefficients"], dtype=np.float64).ravel()[offset: offset + count]
            offset += count
            coefficients = np.minimum(np.maximum(given.reshape(comp.levels.shape), comp.lower), comp.upper)
        else:
            coefficients = np.minimum(np.maximum(comp.centres, comp.lower), comp.upper)
        zetas.append(coefficients)
        xs.append(start_canvas(frame, c, coefficients).astype(dt))
    ps = [(zero(), zero()) for _ in range(C)]
    if start is not None and start.get("p") is not None:
        ps = [(np.asarray(start["p"][c][0], dtype=dt), np.asarray(start["p"][c][1], dtype=dt)) for c in range(C)]
    ws = [(dx_forward(x), dy_forward(x)) for x in xs] if p.tgv else []
    rs = [(zero(), zero(), zero()) for _ in range(C)] if p.tgv else []
    if p.tgv and start is not None and start.get("w") is not None:
        ws = [(np.asarray(start["w"][c][0], dtype=dt), np.asarray(start["w"][c][1], dtype=dt)) for c in range(C)]
    if p.tgv and start is not None and start.get("r") is not None:
        rs = [tuple(np.asarray(start["r"][c][k], dtype=dt) for k in range(3)) for c in range(C)]
    ps = _project(ps, p.alpha1 if p.tgv else p.alpha, p.coupled, False)
    if p.tgv:
        rs = _project(rs, p.alpha0, p.coupled, True)
    state = State(xs, ps, ws, rs)
    tilde = State([x.copy() for x in xs], list(ps), list(ws), list(rs))
    samples = C * frame.rows * frame.columns
    records = []
    stop = 0

    def take(iteration: int) -> bool:
        nonlocal stop
        record = _record(frame, p, tilde, zetas, iteration)
        records.append(record)
        gap = record[1] - record[2]
        met = (p.tolerance > 0 and gap / samples <= p.tolerance) or (
            p.relative_tolerance > 0 and gap <= p.relative_tolerance * record[1]) or (
            p.partial_tolerance > 0 and not math.isnan(record[4]) and record[4] / samples <= p.partial_tolerance)
        if met:
            stop = 1
            return True
        if observer is not None and len(records) > 1 and observer(record, tilde.x):
            stop = 3
            return True
        return False

    stopped = False
    if p.record_every > 0 or p.iterations == 0:
        stopped = take(0)
    n = 0
    rho = dt.type(p.relaxation)
    rest = dt.type(1.0 - p.relaxation)
    while not stopped and n < p.iterations:
        tilde, zetas = _iterate(frame, p, state, dt, rho, rest)
        n += 1
        if (p.record_every > 0 and n % p.record_every == 0) or n == p.iterations:
            stopped = take(n)
    canvas = np.stack([x.astype(np.float64) for x in tilde.x])
    return Solved(canvas, [np.asarray(z, dtype=np.float64) for z in zetas], records, n, stop if stopped else 2)


def _iterate(frame: Frame, p: Plan, s: State, dt, rho, rest):
    """cpp/src/primal_dual.hpp:525-735: one iteration; s is relaxed in place; returns the tilde
    point and the coefficients of its canvas."""
    C = len(frame.components)
    tau, sigma = p.tau, p.sigma
    xt, zetas, wt = [], [], []
    for c in range(C):
        descent = dt.type(tau * p.weights[c])
        v = s.x[c] + descent * divergence(*s.p[c])
        x_tilde, zeta = prox_channel(v, tau, frame.components[c], dt)
        xt.append(x_tilde)
        zetas.append(zeta)
        if p.tgv:
            d1, d2 = div2(*s.r[c])
            wt.append((s.w[c][0] + descent * (s.p[c][0] + d1), s.w[c][1] + descent * (s.p[c][1] + d2)))
    steps_p, steps_r = [], []
    two = dt.type(2.0)
    for c in range(C):
        ascent = dt.type(sigma * p.weights[c])
        bar = two * xt[c] - s.x[c]
        gx, gy = dx_forward(bar), dy_forward(bar)
        if p.tgv:
            wb1 = two * wt[c][0] - s.w[c][0]
            wb2 = two * wt[c][1] - s.w[c][1]
            steps_p.append((s.p[c][0] + ascent * (gx - wb1), s.p[c][1] + ascent * (gy - wb2)))
            e11, e22, e12 = sym_gradient(wb1, wb2)
            steps_r.append((s.r[c][0] + ascent * e11, s.r[c][1] + ascent * e22, s.r[c][2] + ascent * e12))
        else:
            steps_p.append((s.p[c][0] + ascent * gx, s.p[c][1] + ascent * gy))
    pt = _project(steps_p, p.alpha1 if p.tgv else p.alpha, p.coupled, False)
    rt = _project(steps_r, p.alpha0, p.coupled, True) if p.tgv else []
    for c in range(C):
        s.x[c] = rho * xt[c] + rest * s.x[c]
        s.p[c] = (rho * pt[c][0] + rest * s.p[c][0], rho * pt[c][1] + rest * s.p[c][1])
        if p.tgv:
            s.w[c] = (rho * wt[c][0] + rest * s.w[c][0], rho * wt[c][1] + rest * s.w[c][1])
            s.r[c] = tuple(rho * rt[c][k] + rest * s.r[c][k] for k in range(3))
    return State(xt, pt, wt, rt), zetas


def _record(frame: Frame, p: Plan, t: State, zetas, iteration: int):
    """cpp/src/primal_dual.hpp:446-501: primal, dual, TGV's scaling and partial gap, in binary64."""
    C = len(frame.components)
    x = [a.astype(np.float64) for a in t.x]
    data = sum(float(np.sum(value_terms(zetas[c], frame.components[c]))) for c in range(C))
    nan = float("nan")
    squares = 0.0
    first = 0.0
    for c in range(C):
        gx, gy = dx_forward(x[c]), dy_forward(x[c])
        if p.tgv:
            gx = gx - t.w[c][0].astype(np.float64)
            gy = gy - t.w[c][1].astype(np.float64)
        if p.coupled:
            squares = squares + p.weights[c] ** 2 * (gx * gx + gy * gy)
        else:
            first += float(np.sum(p.weights[c] * np.sqrt(gx * gx + gy * gy)))
    if p.coupled:
        first = float(np.sum(np.sqrt(squares)))
    if not p.tgv:
        primal = p.alpha * first + data
        dual = -sum(conjugate(frame, c, p.weights[c] * divergence(*(a.astype(np.float64) for a in t.p[c])),
                              p.free_radius) for c in range(C))
        return (iteration, primal, dual, nan, nan)
    second = 0.0
    squares = 0.0
    d2 = []
    most_square = 0.0
    for c in range(C):
        w1, w2 = (a.astype(np.float64) for a in t.w[c])
        e11, e22, e12 = sym_gradient(w1, w2)
        norm2 = e11 * e11 + e22 * e22 + 2 * (e12 * e12)
        if p.coupled:
            squares = squares + p.weights[c] ** 2 * norm2
        else:
            second += float(np.sum(p.weights[c] * np.sqrt(norm2)))
        d = div2(*(a.astype(np.float64) for a in t.r[c]))
        d2.append(d)
    if p.coupled:
        second = float(np.sum(np.sqrt(squares)))
        most = float(np.max(np.sqrt(sum(d[0] * d[0] + d[1] * d[1] for d in d2))))
    else:
        most = max(float(np.max(np.sqrt(d[0] * d[0] + d[1] * d[1]))) for d in d2)
    del most_square
    primal = (p.alpha1 * first + p.alpha0 * second) + data
    theta = p.alpha1 / most if most > p.alpha1 else 1.0
    dual = -sum(conjugate(frame, c, p.weights[c] * divergence(-theta * d2[c][0], -theta * d2[c][1]), p.free_radius)
                for c in range(C))
    partial = nan
    if p.partial_radius is not None:
        conj = sum(conjugate(frame, c, p.weights[c] * divergence(*(a.astype(np.float64) for a in t.p[c])),
                             p.free_radius) for c in range(C))
        residual = sum(p.weights[c] * float(np.sum(np.sqrt((t.p[c][0] + d2[c][0]) ** 2 + (t.p[c][1] + d2[c][1]) ** 2)))
                       for c in range(C))
        partial = primal + conj + p.partial_radius * residual
    return (iteration, primal, dual, theta, partial)


def options_to_call(options: list[str]) -> tuple[str, dict, list[DataTerm]]:
    """The method, the plan's keywords and the data terms of a list of command-line options
    (the subset the tests use; docs/cli.md:182-243)."""
    values: dict[str, str] = {}
    flags: set[str] = set()
    i = 0
    while i < len(options):
        name = options[i][2:]
        if "=" in name:
            key, value = name.split("=", 1)
            values[key] = value
        elif name in ("no-weight-scaling",):
            flags.add(name)
        else:
            values[name] = options[i + 1]
            i += 1
        i += 1
    method = values.get("method", "tgv")
    number = lambda key: float(values[key]) if key in values else None  # noqa: E731
    keywords = {
        "alpha": number("alpha") or 1.0, "alpha1": number("alpha1") or 1.0, "alpha0": number("alpha0") or 2.0,
        "iterations": int(values["iterations"]) if "iterations" in values else None, "tolerance": number("tolerance"),
        "step_ratio": number("step-ratio"), "step_product": number("step-product") or 0.99,
        "norm_squared": number("norm-squared"),
        "relaxation": number("relaxation") if "relaxation" in values else 1.9,
        "record_every": int(values.get("record-every", 10)), "weight_scaling": "no-weight-scaling" not in flags,
        "channel_weights": [float(v) for v in values["channel-weights"].split(",")] if "channel-weights" in values else None,
        "coupled": values.get("channels", "coupled") == "coupled", "partial_radius": number("partial-radius"),
        "free_radius": number("free-radius") if "free-radius" in values else 255.0,
        "relative_tolerance": number("relative-tolerance") or 0.0,
        "partial_tolerance": number("partial-tolerance") or 0.0,
    }

    def listed(key, convert, default):
        if key not in values:
            return None
        return [convert(v) for v in values[key].split(",")]

    fields = {"mu": listed("mu", lambda v: None if v == "rule" else float(v), None),
              "mu_scale": listed("mu-scale", float, None), "mu_power": listed("mu-power", float, None),
              "mu_chroma": listed("mu-chroma", float, None), "power": listed("weight-power", float, None),
              "dc_weight": listed("dc-weight", float, None), "centres": listed("centres", str, None),
              "slack": listed("slack", float, None), "slack_cost": listed("slack-cost", float, None),
              "flat_weight": listed("flat-weight", float, None), "flat_levels": listed("flat-levels", int, None),
              "flat_dc": listed("flat-dc", lambda v: None if v == "any" else int(v), None)}
    count = max([len(v) for v in fields.values() if v] + [1])
    data = []
    for c in range(count):
        term = DataTerm()
        for key, value in fields.items():
            if value is not None:
                setattr(term, key, value[0] if len(value) == 1 else value[c])
        if method == "mmse":
            term.centres = "mmse"
        data.append(term)
    return method, keywords, data


def run(height: int, width: int, color_space: int, components, options: list[str], *, dtype=np.float64,
        start: dict | None = None) -> Solved:
    """The reconstruction of components [(levels, table, h, v)] with command-line options."""
    method, keywords, data = options_to_call(options)
    frame = make_frame(height, width, color_space, components, data)
    if method == "mmse":
        coefficients = [np.minimum(np.maximum(c.centres, c.lower), c.upper) for c in frame.components]
        canvas = np.stack([start_canvas(frame, c, coefficients[c]) for c in range(len(coefficients))])
        return Solved(canvas, coefficients, [], 0, 0)
    p = plan(method == "tgv", len(frame.components), **keywords)
    return solve(frame, p, dtype=dtype, start=start)
