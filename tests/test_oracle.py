"""The oracle pinned to the reference's golden vectors: the reference's own C++ solver, compiled
in place (oracle/_ref), reproduces every conformance case of the hot path within the case's
binary64 tolerances, with the intervals, weights and steps to the last bit."""

import numpy as np
import pytest

from conftest import case_image, case_options, case_start, golden_cases
from oracle import reference

pytestmark = pytest.mark.skipif(not reference.available(), reason="oracle/_ref is not built (make -C oracle/ref)")


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.stem)
def test_reference_reproduces_golden(path):
    case = np.load(path)
    image = case_image(case)
    components = [(c.coefficients, c.quant_table.reshape(64), c.h_samp_factor, c.v_samp_factor) for c in image.components]
    solved = reference.solve(image.height, image.width, int(image.color_space), components,
                             case_options(case) + ["--threads", "2"], case_start(case))
    assert np.linalg.norm(solved.canvas - case["canvas"]) <= float(case["tolerance_canvas"])
    for index in range(len(components)):
        np.testing.assert_array_equal(solved.lower[index], case[f"lower_{index}"])
        np.testing.assert_array_equal(solved.upper[index], case[f"upper_{index}"])
        np.testing.assert_array_equal(solved.weights[index], case[f"weights_{index}"])
    if "steps" in case.files:
        assert (solved.tau, solved.sigma) == tuple(case["steps"])
    if "records" in case.files:
        records = case["records"]
        assert list(solved.record_iterations) == [int(r) for r in records[:, 0]]
        tolerances = case["record_tolerances"]
        assert np.all(np.abs(solved.records[:, 1] - records[:, 1]) <= tolerances[:, 1])
        assert solved.iterations == int(case["stop_iterations"])
