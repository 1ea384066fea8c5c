"""pic_shutdown frees the top-level workspace and trims the memory pool; a
fresh pic_init afterwards computes the same digits (runs after the other
tests that use the library stream, which it replaces; only the
allocation-free product's file is collected after it)."""
from __future__ import annotations

import hashlib

import pytest

pytestmark = pytest.mark.gpu


def test_pi_after_shutdown_and_reinit(pic, golden):
    torch = pytest.importorskip("torch")
    text1, _ = pic.pi_hex(1_000_000, pic.PI_CHOSEN)
    pic.check(pic.lib().pic_shutdown())
    free_after, _ = torch.cuda.mem_get_info()
    pic.init(0)
    text2, _ = pic.pi_hex(1_000_000, pic.PI_CHOSEN)
    assert text1 == text2
    assert hashlib.md5(text2).hexdigest() == golden["pi"]["1000000"]["md5"]
    # the reserved pool went back to the device: most of it is free again
    _, total = torch.cuda.mem_get_info()
    assert free_after > total // 2
