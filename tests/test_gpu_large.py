"""The large single solve at full size: an 8192x8192 greyscale picture with a custom table of
steps drawn from 1..64, TGV alpha0 = 3, alpha1 = 1.5, 1000 iterations, the primal-dual gap
recorded every 50 iterations. Its parity with the reference's solver is tested at a reduced size
(tests/test_gpu_oracle.py, config5-tgv-custom-reduced); here: every coefficient of all 1,048,576
blocks lies inside its quantization interval in binary64, the records come at 0, 50, ..., 1000
with finite values, the gap shrinks, and the canvas is finite."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPTIONS = ["--method", "tgv", "--alpha1", "1.5", "--alpha0", "3", "--iterations", "1000", "--tolerance", "0",
           "--record-every", "50"]


def test_large_single_solve():
    from unround import native, synthetic

    image = synthetic.large().image
    decoded = native.solve(image, OPTIONS)
    assert decoded.canvas.shape == (1, 8192, 8192)
    assert np.isfinite(decoded.canvas).all()
    zeta = decoded.coefficients[0].reshape(-1)
    assert zeta.size == 1024 * 1024 * 64
    lower = native.model(image, OPTIONS, 0, 0)
    upper = native.model(image, OPTIONS, 0, 1)
    assert np.all(zeta >= lower) and np.all(zeta <= upper)
    history = decoded.result.history
    np.testing.assert_array_equal(history.iterations, np.arange(0, 1001, 50))
    assert np.isfinite(history.primal).all() and np.isfinite(history.dual).all()
    gap = history.gap
    assert gap[-1] < gap[1] and (gap > 0).all()
    assert decoded.result.iterations == 1000
