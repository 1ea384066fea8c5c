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


def test_pi_precision_selected_form_counts_fft_products(pic, golden):
    """The precision-selected form with the FP64 FFT serving every product up
    to 4 M words (the binary-splitting top levels and the Newton steps):
    pi.txt is still the reference's, the statistics report the products and
    the FFT's largest rounding distance; with the acceptance threshold at 0
    every FFT product is recomputed with the NTT and the text is unchanged."""
    saved_fft = pic.get_tuning(pic.TUNE_MUL_FFT_MAX)
    saved_acc = pic.get_tuning(pic.TUNE_FFT_ACCEPT_PPM)
    try:
        pic.set_tuning(pic.TUNE_MUL_FFT_MAX, 1 << 22)
        text, st = pic.pi_hex(1_000_000, pic.PI_CHOSEN)
        assert hashlib.md5(text).hexdigest() == golden["pi"]["1000000"]["md5"]
        assert st["products"] > 0
        assert 0.0 < st["fft_max_err"] < 0.25
        assert st["fft_recomputes"] == 0
        pic.set_tuning(pic.TUNE_FFT_ACCEPT_PPM, 0)
        text, st = pic.pi_hex(100_000, pic.PI_CHOSEN)
        assert hashlib.md5(text).hexdigest() == golden["pi"]["100000"]["md5"]
        assert st["fft_recomputes"] > 0
    finally:
        pic.set_tuning(pic.TUNE_MUL_FFT_MAX, saved_fft)
        pic.set_tuning(pic.TUNE_FFT_ACCEPT_PPM, saved_acc)


@pytest.mark.slow
def test_pi_1e9_two_forms_cross_checked(pic, golden):
    """Pi to 1e9 digits twice: the NTT-only form and the precision-selected
    form (FP64 FFT for every product up to 4 M words where its proven piece
    width allows -- the early Newton steps); both texts equal the reference's
    pi.txt and each other."""
    saved = pic.get_tuning(pic.TUNE_MUL_FFT_MAX)
    try:
        pic.set_tuning(pic.TUNE_MUL_FFT_MAX, 0)
        t1, s1 = pic.pi_hex(1_000_000_000, pic.PI_CHOSEN)
        pic.set_tuning(pic.TUNE_MUL_FFT_MAX, 1 << 22)
        t2, s2 = pic.pi_hex(1_000_000_000, pic.PI_CHOSEN)
    finally:
        pic.set_tuning(pic.TUNE_MUL_FFT_MAX, saved)
    g = golden["pi"]["1000000000"]["md5"]
    assert hashlib.md5(t1).hexdigest() == g
    assert t1 == t2
    assert s1["fft_max_err"] == 0.0 and 0.0 < s2["fft_max_err"] < 0.25


@pytest.mark.parametrize("digits", [1_000_000, 10_000_000])
def test_newton_reuses_the_iterate_transform(pic, golden, digits):
    """The division's and the inverse square root's Newton steps multiply by
    their iterate twice (BigFloat.cpp:510, 561-567); the iterate's forward
    transform is made once per step and reused, and the text is unchanged."""
    text, st = pic.pi_hex(digits, pic.PI_CHOSEN)
    assert hashlib.md5(text).hexdigest() == golden["pi"][str(digits)]["md5"]
    assert st["transform_reuses"] > 0
