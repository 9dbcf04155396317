"""Writes the golden fixtures of tests/golden/ from the reference's conformance cases.

The reference keeps 17 fixed cases (conformance/cases/*.txt of JPEG-Unround, format in
conformance/README.md:55-89): the quantized levels and tables of a small picture, the
options of its reconstruction, and what the reference made of them -- the intervals,
weights and steps to the last bit, the records, the final canvas -- with the tolerances
that bound the rounding of two implementations (docs/math.md, 9). This script reads them
where the reference checkout lies and keeps, for each case on the hot path (the methods
mmse, tv and tgv; the subgradient case is a comparison method outside it), the arrays the
tests compare with, in one compressed .npz per case. The tests read only the .npz files,
so they run where the reference is not present.

Run: python tests/golden/make_golden.py <path to the reference checkout>
(or with the environment variable UNROUND_REFERENCE naming it)
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _floats(items: list[str]) -> np.ndarray:
    return np.array([float(item) for item in items], dtype=np.float64)


def parse_case(path: Path) -> dict[str, np.ndarray]:
    """The arrays of one case file, keyed as the tests read them."""
    lines = [line.split() for line in path.read_text().splitlines() if line and not line.startswith("#")]
    components: dict[int, tuple[int, int, int, int]] = {}
    tables: dict[int, np.ndarray] = {}
    levels: dict[int, dict[int, list[int]]] = {}
    per_block: dict[str, dict[int, dict[int, np.ndarray]]] = {"lower": {}, "upper": {}, "centres": {}, "first-coefficients": {}}
    weights: dict[int, np.ndarray] = {}
    fields: dict[str, dict[tuple[int, int], dict[int, np.ndarray]]] = {"first-p": {}, "first-w": {}, "first-r": {}}
    canvas: dict[int, dict[int, np.ndarray]] = {}
    records: list[list[float]] = []
    record_tolerances: list[list[float]] = []
    out: dict[str, np.ndarray] = {}
    for words in lines:
        key = words[0]
        if key == "name":
            out["name"] = np.array(words[1])
        elif key == "picture":
            out["picture"] = np.array([int(words[1]), int(words[2])], dtype=np.int64)
            out["color_space"] = np.array({"grayscale": 1, "ycbcr": 2, "rgb": 3}[words[3]], dtype=np.int64)
        elif key == "component":
            index, h, v, rows, columns = (int(word) for word in words[1:6])
            components[index] = (h, v, rows, columns)
        elif key == "table":
            tables[int(words[1])] = np.array([int(word) for word in words[2:]], dtype=np.uint16)
        elif key == "levels":
            levels.setdefault(int(words[1]), {})[int(words[2])] = [int(word) for word in words[3:]]
        elif key in per_block:
            per_block[key].setdefault(int(words[1]), {})[int(words[2])] = _floats(words[3:])
        elif key == "weights":
            weights[int(words[1])] = _floats(words[2:])
        elif key in fields:
            entry, channel, row = int(words[1]), int(words[2]), int(words[3])
            fields[key].setdefault((channel, entry), {})[row] = _floats(words[4:])
        elif key == "options":
            out["options"] = np.array(words[1:])
        elif key == "steps":
            out["steps"] = _floats(words[1:3])
        elif key == "record":
            records.append([float(word) for word in words[1:6]])
        elif key == "canvas":
            canvas.setdefault(int(words[1]), {})[int(words[2])] = _floats(words[3:])
        elif key == "stop":
            out["stop_iterations"] = np.array(int(words[1]), dtype=np.int64)
            out["stop_reason"] = np.array(words[2])
        elif key == "tolerance" and words[1] == "canvas":
            out["tolerance_canvas"] = np.array(float(words[2]))
        elif key == "tolerance" and words[1] == "record":
            record_tolerances.append([float(word) for word in words[2:6]])
    count = len(components)
    out["components"] = np.array([components[c] for c in range(count)], dtype=np.int64)
    out["tables"] = np.stack([tables[c] for c in range(count)])
    for c in range(count):
        h, v, rows, columns = components[c]
        rows_of = levels[c]
        out[f"levels_{c}"] = np.array([rows_of[by] for by in range(rows)], dtype=np.int16).reshape(rows, columns, 8, 8)
        for key, values in per_block.items():
            if c in values:
                name = key.replace("-", "_")
                out[f"{name}_{c}"] = np.stack([values[c][by] for by in range(rows)]).reshape(rows, columns, 8, 8)
        if c in weights:
            out[f"weights_{c}"] = weights[c].reshape(8, 8)
    if canvas:
        out["canvas"] = np.stack([np.stack([canvas[c][i] for i in range(len(canvas[c]))]) for c in range(len(canvas))])
    for key, values in fields.items():
        if not values:
            continue
        channels = 1 + max(channel for channel, _ in values)
        entries = 1 + max(entry for _, entry in values)
        name = key.replace("-", "_")
        out[name] = np.stack(
            [
                np.stack([np.stack([values[(c, e)][i] for i in range(len(values[(c, e)]))]) for e in range(entries)])
                for c in range(channels)
            ]
        )
    if records:
        out["records"] = np.array(records, dtype=np.float64)
    if record_tolerances:
        out["record_tolerances"] = np.array(record_tolerances, dtype=np.float64)
    return out


def main() -> None:
    named = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UNROUND_REFERENCE")
    if not named:
        raise SystemExit("name the reference checkout: make_golden.py <path>, or UNROUND_REFERENCE=<path>")
    reference = Path(named)
    cases = sorted((reference / "conformance" / "cases").glob("*.txt"))
    written = 0
    for path in cases:
        case = parse_case(path)
        method = str(case["options"][list(case["options"]).index("--method") + 1])
        if method not in ("mmse", "tv", "tgv"):
            continue
        np.savez_compressed(HERE / f"{path.stem}.npz", **case)
        written += 1
    print(f"wrote {written} fixtures into {HERE}")


if __name__ == "__main__":
    main()
