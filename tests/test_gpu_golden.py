"""The CUDA path against the reference's conformance cases (golden fixtures), through the C
interface. The iterations compute in binary32, the cases in binary64 within tolerances of
binary64 rounding; the bar here is the parity bar: relative L2 <= 1e-4 and max |difference|
<= 2e-3 (0..255 scale) of the canvas, the same records and stop, every coefficient within its
interval in binary64, every record (primal and dual values, TGV's scaling and partial gap)
within 1e-4 of the case's relative to the record's scale, and the decoder of the centres
(binary64 end to end) within the case's own tolerance."""

import numpy as np
import pytest

from conftest import canvas_figures, case_image, case_options, case_start, golden_cases, report_parity
from test_gpu_oracle import RECORDS, record_differences

pytestmark = pytest.mark.gpu

REL_L2 = 1e-4
MAX_ABS = 2e-3


def _dct_blocks(canvas: np.ndarray, rows: int, columns: int, cell: tuple[int, int]) -> np.ndarray:
    """The binary64 coefficients A x of a channel: the DCT of the cell means over its blocks."""
    from unround.synthetic import BASIS

    down, across = cell
    h, w = 8 * rows * down, 8 * columns * across
    means = canvas[:h, :w].reshape(8 * rows, down, 8 * columns, across).mean(axis=(1, 3))
    blocks = means.reshape(rows, 8, columns, 8).transpose(0, 2, 1, 3)
    return np.einsum("kn,abnm,lm->abkl", BASIS, blocks, BASIS)


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: p.stem)
def test_golden_case(path):
    from unround import native

    case = np.load(path)
    image = case_image(case)
    decoded = native.solve_from(image, case_options(case), start=case_start(case))
    expected = case["canvas"]
    assert decoded.canvas.shape == expected.shape
    difference = decoded.canvas - expected
    method = case_options(case)[case_options(case).index("--method") + 1]
    if method == "mmse":
        assert np.linalg.norm(difference) <= float(case["tolerance_canvas"])
        assert decoded.result is None
        return
    figures = canvas_figures(decoded.canvas, expected)
    # Records at the same iterations: primal and dual values, TGV's scaling and partial gap.
    records = case["records"]
    history = decoded.result.history
    worst = record_differences(history, [int(r) for r in records[:, 0]], records)
    report_parity(f"golden {path.stem}", **figures, **{f"record_{k}": v for k, v in worst.items()})
    assert figures["rel_l2"] <= REL_L2, figures
    assert figures["max_abs"] <= MAX_ABS, figures
    assert max(worst.values()) <= RECORDS, worst
    np.testing.assert_allclose(history.primal, records[:, 1], rtol=2e-5)
    assert decoded.result.iterations == int(case["stop_iterations"])
    assert decoded.result.stop.name.lower() == str(case["stop_reason"])
    # Every coefficient within its interval, in binary64, to 1e-4 of its step (docs/math.md 1.2).
    for index, problem in enumerate(decoded.problems):
        coefficients = decoded.coefficients[index]
        q = problem.steps[None, None]
        assert np.all(coefficients >= problem.lower - 1e-9) and np.all(coefficients <= problem.upper + 1e-9)
        np.testing.assert_array_equal(problem.lower, case[f"lower_{index}"])
        np.testing.assert_array_equal(problem.upper, case[f"upper_{index}"])
        np.testing.assert_array_equal(problem.steps.ravel(), case["tables"][index].astype(np.float64))
        np.testing.assert_array_equal(problem.weights, case[f"weights_{index}"])
        a = _dct_blocks(decoded.canvas[index], coefficients.shape[0], coefficients.shape[1], problem.ratio)
        assert np.all(a >= problem.lower - 1e-4 * q) and np.all(a <= problem.upper + 1e-4 * q)
