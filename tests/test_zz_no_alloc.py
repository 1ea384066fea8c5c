"""pic_mul_noalloc -- the product for callers that cannot allocate device
memory when they multiply (an application whose device memory already belongs
to its own pool allocator, or a latency-critical loop that must not take the
allocator's locks or risk running out of memory mid-computation).

It runs the three-prime NTT in fixed storage compiled into the library, so
its words must equal those of pic_mul, the allocating entry point, exactly
(products are integers: the tolerance is zero).  Two calls in a row check that
the shared storage carries nothing over from the previous call.  The
library's allocation counter (every pool allocation, every direct cudaMalloc
of a twiddle table, pinned staging) must not move during a call, including a
first call at a length no other entry point has used yet.  This file is
collected last so that a run stopping at its first failure has already run
every other test."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.ffi import random_words

pytestmark = pytest.mark.gpu

CASES = [(1, 1), (7, 3), (1000, 2500), (20000, 30000), (65536, 65538)]


def _dev(torch, w):
    return torch.from_numpy(np.ascontiguousarray(w).view(np.int32)).cuda()


def _noalloc(pic, torch, z, ta, na, tb, nb):
    """One pic_mul_noalloc call; asserts that the library allocated nothing."""
    L = pic.lib()
    s = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    held, count = L.pic_device_bytes_in_use(), L.pic_debug_allocation_count()
    pic.check(L.pic_mul_noalloc(z.data_ptr(), ta.data_ptr(), na, tb.data_ptr(), nb, s))
    torch.cuda.synchronize()
    assert L.pic_device_bytes_in_use() == held
    assert L.pic_debug_allocation_count() == count, "pic_mul_noalloc allocated"


def test_noalloc_first_call_at_a_fresh_length(pic, torch_cuda):
    """Before pic_mul has run at this length (no tables or buffers of its size
    exist yet), the no-allocation product still allocates nothing."""
    torch = torch_cuda
    na, nb = 40001, 24999
    a, b = random_words(901, na), random_words(902, nb)
    ta, tb = _dev(torch, a), _dev(torch, b)
    z = torch.full((na + nb,), -1, dtype=torch.int32, device="cuda")
    _noalloc(pic, torch, z, ta, na, tb, nb)
    want = int.from_bytes(a.tobytes(), "little") * int.from_bytes(b.tobytes(), "little")
    got = int.from_bytes(z.cpu().numpy().view(np.uint32).tobytes(), "little")
    assert got == want


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
        _noalloc(pic, torch, z_new, ta, na, tb, nb)
        assert torch.equal(z_new, z_ref), f"call {call}: products differ"


@pytest.mark.parametrize("n", [5, 3000, 65536])
def test_noalloc_squaring_same_pointer(pic, torch_cuda, n):
    """a and b the same device pointer: the squaring branch transforms once."""
    torch = torch_cuda
    L = pic.lib()
    s = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        ta = _dev(torch, random_words(70 + n + call, n))
        z_ref = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
        z_new = torch.full((2 * n,), -1, dtype=torch.int32, device="cuda")
        pic.check(L.pic_mul(z_ref.data_ptr(), ta.data_ptr(), n, ta.data_ptr(), n, pic.MUL_NTT3, s))
        _noalloc(pic, torch, z_new, ta, n, ta, n)
        assert torch.equal(z_new, z_ref), f"call {call}: squares differ"


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
