"""Whole pi runs: pi.txt byte for byte against the reference's own output."""
from __future__ import annotations

import hashlib

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("digits", [10_000, 100_000, 1_000_000])
@pytest.mark.parametrize("form", ["chosen", "plain"])
def test_pi_matches_reference(pic, golden, digits, form):
    if form == "plain" and digits > 100_000:
        pytest.skip("plain form at 1M digits is covered by the benchmark")
    text, st = pic.pi_hex(digits, pic.PI_CHOSEN if form == "chosen" else pic.PI_PLAIN)
    g = golden["pi"][str(digits)]
    assert len(text) == g["bytes"]
    assert text[:80].decode() == g["head"]
    assert text[-80:].decode() == g["tail"]
    assert hashlib.md5(text).hexdigest() == g["md5"]
    assert st["terms"] > 0 and st["kernel_launches"] > 0


@pytest.mark.slow
@pytest.mark.parametrize("digits", [10_000_000, 100_000_000, 1_000_000_000])
def test_pi_large_matches_reference(pic, golden, digits):
    """Up to the full 1e9-digit run: every hex digit equal to the reference's
    pi.txt (the 1e9 fixture is the reference program's own 8-thread run)."""
    text, st = pic.pi_hex(digits, pic.PI_CHOSEN)
    g = golden["pi"][str(digits)]
    assert len(text) == g["bytes"]
    assert text[:80].decode() == g["head"]
    assert text[-80:].decode() == g["tail"]
    assert hashlib.md5(text).hexdigest() == g["md5"]


@pytest.mark.parametrize("digits", [3_141_593, 27_182_818])
def test_pi_odd_sizes_match_reference(pic, golden, digits):
    """Digit counts that are not powers of ten: other term counts, working
    precisions and top-level merge shapes, pi.txt equal to the reference's."""
    text, _ = pic.pi_hex(digits, pic.PI_CHOSEN)
    g = golden["pi"][str(digits)]
    assert len(text) == g["bytes"]
    assert text[-80:].decode() == g["tail"]
    assert hashlib.md5(text).hexdigest() == g["md5"]


def test_pi_oracle_agrees_small(pic, oracle):
    text, _ = pic.pi_hex(20_000, pic.PI_CHOSEN)
    assert text == oracle.pi_hex(20_000)
