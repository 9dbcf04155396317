"""Test configuration: the package and the oracle on the path, and the gpu marker.

Tests marked gpu run on a B200 (`pytest -m gpu`); the others need no GPU (`-m "not gpu"`).
The oracle (oracle/) is test infrastructure: the tests use it as the checker only.
"""

import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for path in (ROOT / "jpeg-unround_b200", ROOT):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a B200 (CUDA device)")


# Parity figures of the GPU tests against the reference's solver: one dict per case, printed at
# the end of the run and, where UNROUND_PARITY_REPORT names a file, written there as JSON.
PARITY: list[dict] = []


def report_parity(case: str, **figures) -> None:
    PARITY.append({"case": case, **{k: (float(v) if hasattr(v, "__float__") else v) for k, v in figures.items()}})


def canvas_figures(ours: np.ndarray, theirs: np.ndarray) -> dict[str, float]:
    """Relative L2 and max |difference| of two canvases (0..255 scale)."""
    difference = ours - theirs
    return {"rel_l2": float(np.linalg.norm(difference) / np.linalg.norm(theirs)),
            "max_abs": float(np.max(np.abs(difference)))}


def pytest_terminal_summary(terminalreporter, exitstatus, config) -> None:
    if not PARITY:
        return
    terminalreporter.section("parity against the reference's solver")
    for entry in PARITY:
        terminalreporter.write_line(
            " ".join(f"{k}={v:.3g}" if isinstance(v, float) else f"{k}={v}" for k, v in entry.items()))
    target = os.environ.get("UNROUND_PARITY_REPORT")
    if target:
        Path(target).parent.mkdir(parents=True, exist_ok=True)
        Path(target).write_text(json.dumps(PARITY, indent=1))


def golden_cases() -> list[Path]:
    return sorted(GOLDEN.glob("*.npz"))


def case_image(case: np.lib.npyio.NpzFile):
    """The unround.jpegio.Image of a golden case."""
    from unround import jpegio

    components = []
    for c in range(len(case["components"])):
        h, v, _, _ = (int(x) for x in case["components"][c])
        components.append((case[f"levels_{c}"], case["tables"][c], h, v))
    height, width = (int(x) for x in case["picture"])
    return jpegio.image_of(height, width, int(case["color_space"]), components)


def case_start(case: np.lib.npyio.NpzFile) -> dict[str, np.ndarray] | None:
    """The state a one-iteration case starts from, or None."""
    if "first_coefficients_0" not in case.files:
        return None
    count = len(case["components"])
    start = {"coefficients": np.concatenate([case[f"first_coefficients_{c}"].ravel() for c in range(count)])}
    for name in ("p", "w", "r"):
        if f"first_{name}" in case.files:
            start[name] = case[f"first_{name}"]
    return start


def case_options(case: np.lib.npyio.NpzFile) -> list[str]:
    return [str(option) for option in case["options"]]
