"""unround_b200_decode_centres_noalloc, the decoder of the centres that allocates no device
memory: its output in caller-owned device buffers against unround_solve's with --method=mmse on
the same input, call after call (the scratch array keeps what the last call left there); that a
warm call leaves the device's free memory, its stream-ordered pool and torch's allocator exactly
as they were; and its refusals. The file is named to be collected last, after the tests that load
the library."""

import ctypes

import numpy as np
import pytest

OPTIONS = ["--method", "mmse"]
SCRATCH = 64 << 20
MESSAGE = 1024


def _function():
    from unround import native

    library = native._library()
    function = library.unround_b200_decode_centres_noalloc
    u64 = ctypes.c_uint64
    function.restype = ctypes.c_int32
    function.argtypes = [ctypes.POINTER(native._Input), ctypes.c_void_p, ctypes.c_void_p, u64, ctypes.c_void_p, u64,
                         ctypes.POINTER(u64), ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    return function


def _call(image, canvas=None, coefficients=None, options=OPTIONS, stream=None):
    """(status, message, sizes): canvas and coefficients are device tensors or None (sizes only)."""
    from unround import native

    function = _function()
    settings = native._settings_of(options)
    given, kept = native._input_of(image)
    sizes = (ctypes.c_uint64 * 4)()
    message = ctypes.create_string_buffer(MESSAGE)
    status = function(ctypes.byref(given), settings.handle,
                      None if canvas is None else canvas.data_ptr(), 0 if canvas is None else canvas.numel(),
                      None if coefficients is None else coefficients.data_ptr(),
                      0 if coefficients is None else coefficients.numel(), sizes, stream, message, MESSAGE)
    del kept
    return int(status), message.value.decode(), tuple(int(s) for s in sizes)


def _images():
    from unround import synthetic

    yield "colour420", synthetic.colour(61, 77, quality=75, seed=8, noise=3).image
    yield "grey", synthetic.grey(64, 48, quality=30, seed=4).image
    yield "colour422-large", synthetic.colour(1024, 1536, quality=60, seed=9, sampling=(1, 2)).image


def test_sizes_without_a_device():
    from unround import synthetic

    image = synthetic.colour(61, 77, quality=75, seed=8).image
    status, message, sizes = _call(image)
    assert status == 0, message
    blocks = sum(c.coefficients.shape[0] * c.coefficients.shape[1] for c in image.components)
    assert sizes == (3, 64, 80, 64 * blocks)
    status, message, _ = _call(image, options=["--method", "tgv"])
    assert status == 1 and "--method=mmse" in message


@pytest.mark.gpu
def test_against_unround_solve_call_after_call():
    import torch

    from unround import native

    stream = torch.cuda.current_stream().cuda_stream
    images = list(_images())
    outputs = {}
    for name, image in images + images[:1]:
        expected = native.solve(image, OPTIONS)
        status, message, (channels, rows, columns, count) = _call(image)
        assert status == 0, message
        assert (channels, rows, columns) == expected.canvas.shape
        canvas = torch.full((channels, rows, columns), float("nan"), dtype=torch.float64, device="cuda")
        coefficients = torch.full((count,), float("nan"), dtype=torch.float64, device="cuda")
        status, message, _ = _call(image, canvas, coefficients, stream=stream)
        assert status == 0, message
        got_canvas = canvas.cpu().numpy()
        got_coefficients = coefficients.cpu().numpy()
        # The same kernels on the same inputs: identical to the last bit.
        np.testing.assert_array_equal(got_canvas, expected.canvas, err_msg=name)
        np.testing.assert_array_equal(got_coefficients, np.concatenate([c.reshape(-1) for c in expected.coefficients]),
                                      err_msg=name)
        if name in outputs:
            np.testing.assert_array_equal(got_canvas, outputs[name])
        outputs[name] = got_canvas


def _device_memory():
    """(free bytes of the device, the default pool's reserved and used bytes, torch's reserved and
    allocated bytes): what a device allocation by anyone in this process would change."""
    import torch
    from cuda.bindings import driver

    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    (error,) = driver.cuInit(0)
    assert error == driver.CUresult.CUDA_SUCCESS
    error, device = driver.cuDeviceGet(torch.cuda.current_device())
    assert error == driver.CUresult.CUDA_SUCCESS
    error, pool = driver.cuDeviceGetDefaultMemPool(device)
    assert error == driver.CUresult.CUDA_SUCCESS
    attributes = driver.CUmemPool_attribute
    pooled = []
    for attribute in (attributes.CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT, attributes.CU_MEMPOOL_ATTR_USED_MEM_CURRENT):
        error, value = driver.cuMemPoolGetAttribute(pool, attribute)
        assert error == driver.CUresult.CUDA_SUCCESS
        pooled.append(int(value))
    return (int(free), *pooled, torch.cuda.memory_reserved(), torch.cuda.memory_allocated())


@pytest.mark.gpu
def test_allocates_nothing():
    import torch

    from unround import synthetic

    image = synthetic.colour(517, 389, quality=55, seed=21).image
    status, message, (channels, rows, columns, count) = _call(image)
    assert status == 0, message
    canvas = torch.empty((channels, rows, columns), dtype=torch.float64, device="cuda")
    coefficients = torch.empty(count, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # The first call may load the library's device code (and with it the scratch array).
    status, message, _ = _call(image, canvas, coefficients, stream=stream)
    assert status == 0, message
    first = canvas.clone()
    before = _device_memory()
    for _ in range(2):
        status, message, _ = _call(image, canvas, coefficients, stream=stream)
        assert status == 0, message
        assert _device_memory() == before
    assert torch.equal(canvas, first)


@pytest.mark.gpu
def test_refusals():
    import torch

    from unround import jpegio

    # 750 x 750 blocks: 72 MB of levels, more than the scratch array holds.
    levels = np.zeros((750, 750, 8, 8), dtype=np.int16)
    image = jpegio.image_of(6000, 6000, jpegio.ColorSpace.GRAYSCALE, [(levels, np.full(64, 16), 1, 1)])
    status, message, (channels, rows, columns, count) = _call(image)
    assert status == 0, message
    assert 2 * count > SCRATCH
    small = torch.zeros(8, dtype=torch.float64, device="cuda")
    status, message, _ = _call(image, small, small)
    assert status == 1 and "output buffers" in message
    canvas = torch.zeros((channels, rows, columns), dtype=torch.float64, device="cuda")
    coefficients = torch.zeros(count, dtype=torch.float64, device="cuda")
    status, message, _ = _call(image, canvas, coefficients)
    assert status == 1 and "scratch" in message
    assert not bool(canvas.any()) and not bool(coefficients.any())
