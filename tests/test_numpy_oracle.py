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
