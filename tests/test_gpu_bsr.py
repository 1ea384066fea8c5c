"""Batched binary splitting (bsr.cu) vs the oracle's Pi_BSR restatement:
P, Q, R word for word, through both merge algorithms."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(0, 5, 100), (0, 4, 16), (0, 50, 10_000), (0, 706, 923), (17, 600, 5_000),
         (0, 3000, 200), (0, 2000, 100_000), (1000, 1257, 50), (0, 8000, 300_000)]


def _same(dev, want) -> bool:
    got = dev.to_bf()
    return (got.sign == want.sign and got.exp == want.exp and got.words.size == want.words.size
            and np.array_equal(got.words, want.words))


# (schoolbook threshold, wrapped NTT merges): 8 sends nearly every level
# through the batched NTT merges, with and without wrapped products.
@pytest.mark.parametrize("a,b,p", CASES)
# Small-merge modes: 2 = thread, warp and CTA kernels (by node size), 0 = CTA
# kernel for every schoolbook level.
# Combine: P formed in the transform domain (1) or from two separate products (0).
@pytest.mark.parametrize("school_max,wrap,small,combine", [(192, 1, 2, 1), (192, 1, 0, 1), (8, 1, 2, 1),
                                                           (8, 0, 2, 1), (8, 1, 2, 0)])
# Three-prime form of the NTT merges: integer (0) or FP64 (1).
@pytest.mark.parametrize("form", [0, 1])
def test_bsr_vs_oracle(pic, oracle, a, b, p, school_max, wrap, small, combine, form):
    knobs = {pic.TUNE_BSR_SCHOOL_MAX: school_max, pic.TUNE_BSR_WRAP: wrap, pic.TUNE_BSR_SMALL_MERGE: small,
             pic.TUNE_BSR_COMBINE: combine, pic.TUNE_NTT_FORM: form}
    saved = {k: pic.get_tuning(k) for k in knobs}
    for k, v in knobs.items():
        pic.set_tuning(k, v)
    try:
        P, Q, R = pic.bsr(a, b, p, pic.PI_CHOSEN)
    finally:
        for k, v in saved.items():
            pic.set_tuning(k, v)
    wP, wQ, wR = oracle.bsr(a, b, p)
    assert _same(Q, wQ), "Q"
    assert _same(R, wR), "R"
    assert _same(P, wP), "P"


def test_bsr_plain_form_vs_oracle(pic, oracle):
    P, Q, R = pic.bsr(0, 300, 1000, pic.PI_PLAIN)
    wP, wQ, wR = oracle.bsr(0, 300, 1000)
    assert _same(P, wP) and _same(Q, wQ) and _same(R, wR)


# CTA schoolbook merges with one Karatsuba level (threshold 4, 16, 64 words;
# school_max 600 keeps every level up to 600-word children on the CTA
# kernel), the thread / warp kernels off so the CTA kernel sees short nodes too.
@pytest.mark.parametrize("a,b,p", [(0, 706, 923), (0, 3000, 200), (0, 2000, 100_000), (0, 8000, 300_000)])
@pytest.mark.parametrize("kara", [4, 16, 64])
def test_bsr_karatsuba_vs_oracle(pic, oracle, a, b, p, kara):
    knobs = {pic.TUNE_BSR_SCHOOL_MAX: 600, pic.TUNE_BSR_SMALL_MERGE: 0, pic.TUNE_BSR_KARATSUBA: kara}
    saved = {k: pic.get_tuning(k) for k in knobs}
    for k, v in knobs.items():
        pic.set_tuning(k, v)
    try:
        P, Q, R = pic.bsr(a, b, p, pic.PI_CHOSEN)
    finally:
        for k, v in saved.items():
            pic.set_tuning(k, v)
    wP, wQ, wR = oracle.bsr(a, b, p)
    assert _same(Q, wQ), "Q"
    assert _same(R, wR), "R"
    assert _same(P, wP), "P"
