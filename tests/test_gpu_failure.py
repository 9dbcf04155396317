"""The failure path of the kernels' bounded waits, made to run without a fault or a hang: the
dual sweep's compute warps are given 0 tries for each chunk of their ring
(unround_b200_set_ring_wait_limit), so every CTA gives up at its first chunk although the chunk's
loads complete as usual; the CTA then drains those loads (at the full limit) and leaves. The
solve reports UNROUND_ERROR_INTERNAL with the message of a wait that ran out, and the next solve
on the same device, with the full limit back, succeeds and gives the same canvas as before."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPTIONS = ["--method", "tgv", "--iterations", "12", "--tolerance", "0", "--record-every", "4"]


def _setter():
    from unround import native

    function = native._library().unround_b200_set_ring_wait_limit
    function.restype = ctypes.c_int64
    function.argtypes = [ctypes.c_int64]
    return function


@pytest.mark.parametrize("kind", ["grey", "colour420"])
def test_a_wait_that_runs_out_is_an_internal_error(kind):
    from unround import native, synthetic

    image = (synthetic.grey(64, 96, quality=40, seed=61).image if kind == "grey"
             else synthetic.colour(48, 80, quality=60, seed=62).image)
    before = native.solve(image, OPTIONS)
    set_limit = _setter()
    full = set_limit(0)
    try:
        with pytest.raises(native.UnroundError) as raised:
            native.solve(image, OPTIONS)
    finally:
        assert set_limit(-1) == 0
    assert full == 1 << 22
    assert raised.value.status == native.Status.INTERNAL
    assert "a bounded wait of the sweep ran out" in raised.value.message
    # The device and the library carry on.
    after = native.solve(image, OPTIONS)
    np.testing.assert_array_equal(after.canvas, before.canvas)
    assert set_limit(-1) == 1 << 22
