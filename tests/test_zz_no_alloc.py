"""pic_mul_noalloc -- the product for callers that cannot allocate device
memory when they multiply (an application whose device memory already belongs
to its own pool allocator, or a latency-critical loop that must not take the
allocator's locks or risk running out of memory mid-computation).

It runs the three-prime NTT in fixed storage compiled into the library, so
its words must equal those of pic_mul, the allocating entry point, exactly
(products are integers: the tolerance is zero).  Two calls in a row check that
the shared storage carries nothing over from the previous call, and the
library's device-memory counter must not move during either call.  This file
is collected last so that a run stopping at its first failure has already run
every other test."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.ffi import random_words

pytestmark = pytest.mark.gpu

CASES = [(1, 1), (7, 3), (1000, 2500), (20000, 30000), (65536, 65538)]


def _dev(torch, w):
    return torch.from_numpy(np.ascontiguousarray(w).view(np.int32)).cuda()


@pytest.mark.parametrize("na,nb", CASES)
def test_noalloc_equals_pic_mul_on_two_calls(pic, torch_cuda, na, nb):
    torch = torch_cuda
    L = pic.lib()
    s = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        a = random_words(10 * na + call, na)
        b = random_words(10 * nb + 5 + call, nb)
        ta, tb = _dev(torch, a), _dev(torch, b)
        z_ref = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
        z_new = torch.full((na + nb,), -1, dtype=torch.int32, device="cuda")
        pic.check(L.pic_mul(z_ref.data_ptr(), ta.data_ptr(), na, tb.data_ptr(), nb, pic.MUL_NTT3, s))
        torch.cuda.synchronize()
        held = L.pic_device_bytes_in_use()
        pic.check(L.pic_mul_noalloc(z_new.data_ptr(), ta.data_ptr(), na, tb.data_ptr(), nb, s))
        torch.cuda.synchronize()
        assert L.pic_device_bytes_in_use() == held
        assert torch.equal(z_new, z_ref), f"call {call}: products differ"


def test_noalloc_rejects_products_beyond_its_storage(pic, torch_cuda):
    torch = torch_cuda
    L = pic.lib()
    na, nb = 65536, 65540  # ceil(na/2) + ceil(nb/2) - 1 = 65537 points
    ta = torch.zeros(na, dtype=torch.int32, device="cuda")
    tb = torch.zeros(nb, dtype=torch.int32, device="cuda")
    z = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
    rc = L.pic_mul_noalloc(z.data_ptr(), ta.data_ptr(), na, tb.data_ptr(), nb, None)
    assert rc == pic.ERR_LENGTH
    assert b"65536" in L.pic_last_error()
