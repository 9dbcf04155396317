"""The NumPy restatement of the oracle (oracle/unround_oracle.py) pinned to the reference's
golden vectors: every conformance case of the path within its binary64 tolerance, and its
binary32 mode (the device's arithmetic, DC centred) within the parity bar (relative L2 <= 1e-4,
max |difference| <= 2e-3 on 0..255) of binary64."""

import numpy as np
import pytest

from conftest import case_image, case_options, case_start, golden_cases
from oracle import unround_oracle as oracle


def _components(image):
    return [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor) for c in image.components]


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.stem)
def test_restatement_reproduces_golden(path):
    case = np.load(path)
    image = case_image(case)
    solved = oracle.run(image.height, image.width, int(image.color_space), _components(image), case_options(case),
                        start=case_start(case))
    assert np.linalg.norm(solved.canvas - case["canvas"]) <= float(case["tolerance_canvas"])
    if "records" in case.files:
        records = case["records"]
        assert [r[0] for r in solved.records] == [int(x) for x in records[:, 0]]
        primal = np.array([r[1] for r in solved.records])
        assert np.all(np.abs(primal - records[:, 1]) <= case["record_tolerances"][:, 1])
        assert solved.iterations == int(case["stop_iterations"])


@pytest.mark.parametrize("name", ["grey-tgv", "colour420-tv"])
def test_binary32_mode_within_bar(name):
    case = np.load(next(p for p in golden_cases() if p.stem == name))
    image = case_image(case)
    components = _components(image)
    wide = oracle.run(image.height, image.width, int(image.color_space), components, case_options(case))
    narrow = oracle.run(image.height, image.width, int(image.color_space), components, case_options(case),
                        dtype=np.float32)
    difference = narrow.canvas - wide.canvas
    assert np.linalg.norm(difference) / np.linalg.norm(wide.canvas) <= 1e-4
    assert np.max(np.abs(difference)) <= 2e-3


def test_binary32_iterates_move_the_dual_record():
    """The NumPy restatement of the device's binary32 arithmetic against itself in binary64, on a
    96 x 128 4:2:0 TGV picture for 500 iterations: the canvas and the primal value agree to
    binary32 rounding, but the dual value drifts further, to about 5e-4 of the record's scale at
    500 iterations (the records are binary64 sums from the binary32 tilde point, so this is the
    iterates' drift, not the records' arithmetic). The device's dual records at hundreds of
    iterations are held to the reference's within that drift's order, not within 1e-4."""
    from unround import synthetic

    image = synthetic.colour(96, 128, quality=75, seed=2, noise=3).image
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor)
                  for c in image.components]
    options = ["--method", "tgv", "--iterations", "500", "--tolerance", "0", "--record-every", "100"]
    wide = oracle.run(image.height, image.width, 2, components, options, dtype=np.float64)
    narrow = oracle.run(image.height, image.width, 2, components, options, dtype=np.float32)
    assert np.linalg.norm(narrow.canvas - wide.canvas) / np.linalg.norm(wide.canvas) < 1e-6
    drift = []
    for a, b in zip(wide.records, narrow.records):
        scale = max(abs(a[1]), abs(a[2]))
        assert abs(a[1] - b[1]) / scale < 1e-5  # the primal value
        drift.append(abs(a[2] - b[2]) / scale)
    assert drift[1] < 1e-4 < drift[-1] < 1e-2
