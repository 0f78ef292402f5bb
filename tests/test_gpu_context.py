"""The caller's current CUDA context survives every call, including a custom
context and no context at all (reference tests/test_cuda_context.py:17-71)."""
import ctypes as ct

import numpy as np
import pytest

import harvest_cuda_b200 as hv
from harvest_cuda_b200 import signals

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seconds", [0.3, 2.1])
def test_custom_context_is_restored(gpu, seconds):
    driver = ct.CDLL("libcuda.so.1")
    driver.cuCtxCreate_v2.argtypes = [ct.POINTER(ct.c_void_p), ct.c_uint, ct.c_int]
    driver.cuCtxGetCurrent.argtypes = [ct.POINTER(ct.c_void_p)]
    driver.cuCtxSetCurrent.argtypes = [ct.c_void_p]
    driver.cuCtxDestroy_v2.argtypes = [ct.c_void_p]

    def check(result):
        assert result == 0, f"CUDA driver error {result}"

    def current():
        out = ct.c_void_p()
        check(driver.cuCtxGetCurrent(ct.byref(out)))
        return out.value

    check(driver.cuInit(0))
    x = signals.kind_clip("speechlike", seconds, 16000)
    expected = hv.harvest(x, 16000)
    previous = current()
    custom = ct.c_void_p()
    check(driver.cuCtxCreate_v2(ct.byref(custom), 0, 0))
    try:
        for context in (custom.value, None, custom.value):
            check(driver.cuCtxSetCurrent(context))
            actual = hv.harvest(x, 16000)
            assert current() == context
            for got, want in zip(actual, expected):
                np.testing.assert_array_equal(got, want)
            hv.clear_cache()
            assert current() == context
    finally:
        check(driver.cuCtxSetCurrent(previous))
        check(driver.cuCtxDestroy_v2(custom))
