"""Failure handling without any GPU fault: injected allocation failures,
bad lengths and arguments come back as statuses and leave the library usable."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.ffi import random_words

pytestmark = pytest.mark.gpu


def test_injected_allocation_failure_then_recovery(pic, oracle):
    L = pic.lib()
    a, b = random_words(1, 5000), random_words(2, 5000)
    L.pic_debug_fail_allocations(1)
    with pytest.raises(pic.PicError) as e:
        pic.mul_host(a, b, "ntt3")
    assert e.value.status == pic.ERR_NO_MEMORY
    L.pic_debug_fail_allocations(0)
    assert np.array_equal(pic.mul_host(a, b, "ntt3"), oracle.mul_words(a, b))


def test_bad_arguments(pic, torch_cuda):
    L = pic.lib()
    assert L.pic_mul(None, None, 1, None, 1, 0, None) == pic.ERR_INVALID
    assert L.pic_ntt_forward(None, 12, None) == pic.ERR_INVALID
    t = torch_cuda.zeros(16, dtype=torch_cuda.int64, device="cuda")
    assert L.pic_ntt_forward(t.data_ptr(), 40, None) == pic.ERR_INVALID
    assert L.pic_pi_hex(10, 7, None, 0, None, None) == pic.ERR_INVALID
    z = np.zeros(4, dtype=np.uint32)
    assert L.pic_mul_host(z.ctypes.data, z.ctypes.data, 0, z.ctypes.data, 1, 0) == pic.ERR_INVALID
