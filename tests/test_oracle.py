"""The CPU oracle (oracle/pic_oracle.c) pinned against the reference: golden
fixtures generated from the reference's own code, and -- where the reference
was compiled in this checkout -- the reference harness directly."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle.ffi import BF, MODE_FFT, MODE_NTT, MODE_SCHOOL, MODE_AUTO, random_words, splitmix64_np


def _bf(rec):
    return BF(bool(rec[0]), int(rec[1]), np.array(rec[2], dtype=np.uint32))


def _words_md5(w):
    return hashlib.md5(np.ascontiguousarray(w, dtype="<u4").tobytes()).hexdigest()


def test_pi_sizes_match_pi_h(oracle):
    # PI.h:141-144 for the digit counts the reference was run at
    assert oracle.pi_sizes(1_000_000) == (830_482, 92_276, 70_515)
    assert oracle.pi_sizes(10_000) == (8_304, 923, 706)


@pytest.mark.parametrize("digits", [10_000, 100_000])
def test_oracle_pi_matches_reference_md5(oracle, golden, digits):
    text = oracle.pi_hex(digits)
    g = golden["pi"][str(digits)]
    assert len(text) == g["bytes"]
    assert text[:80].decode() == g["head"]
    assert hashlib.md5(text).hexdigest() == g["md5"]


def test_golden_bigfloat_ops(oracle, golden):
    for rec in golden["bigfloat"]["ops"]:
        a, b, p = _bf(rec["a"]), _bf(rec["b"]), rec["p"]
        for name in ("add", "sub", "mul"):
            assert getattr(oracle, name)(a, b, p).same(_bf(rec[name])), (name, rec)
        assert oracle.rcp(a, p).same(_bf(rec["rcp"]))
        assert oracle.div(a, b, p).same(_bf(rec["div"]))
        s = rec["mul_u32"][0]
        assert oracle.mul_u32(a, s).same(_bf(rec["mul_u32"][1:]))
    for rec in golden["bigfloat"]["invsqrt"]:
        assert oracle.invsqrt(rec["x"], rec["p"]).same(_bf(rec["z"]))
    c = golden["bigfloat"]["carry_loss"]
    assert oracle.add(_bf(c["a"]), _bf(c["b"]), c["p"]).same(_bf(c["add"]))


def test_golden_small_products(oracle, golden):
    for rec in golden["products"]["small"]:
        a = random_words(rec["seed_a"], rec["na"])
        b = random_words(rec["seed_b"], rec["nb"])
        a[-1] |= 1
        b[-1] |= 1
        z = oracle.mul(BF(True, 0, a), BF(True, 0, b))
        assert z.words.tolist() == rec["z"]
        # and against Python's exact integers
        ia = int.from_bytes(a.astype("<u4").tobytes(), "little")
        ib = int.from_bytes(b.astype("<u4").tobytes(), "little")
        assert BF(True, 0, z.words).to_int() == ia * ib


def test_golden_edge_products(oracle, golden):
    for rec in golden["products"]["edge"]:
        n = rec["n"]
        ones = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
        if rec["kind"] == "ones":
            a, b = ones, ones
        else:
            a = np.zeros(n, dtype=np.uint32)
            a[0] = 1
            a[-1] = 1
            b = ones
        z = oracle.mul(BF(True, 0, a), BF(True, 0, b))
        assert z.L == rec["L"] and _words_md5(z.words) == rec["md5"]


@pytest.mark.parametrize("lg", [12, 16])
def test_golden_isolated_products(oracle, golden, lg):
    rec = [r for r in golden["products"]["isolated"] if r["log2n"] == lg][0]
    n = 1 << lg
    z = oracle.mul(BF(True, 0, random_words(42, n)), BF(True, 0, random_words(43, n)))
    assert z.L == rec["L"] and _words_md5(z.words) == rec["md5"]


def test_mul_modes_agree(oracle):
    for n in (1, 5, 64, 333, 2000):
        a = random_words(11 + n, n)
        b = random_words(12 + n, n + 7)
        outs = []
        for mode in (MODE_SCHOOL, MODE_FFT, MODE_NTT, MODE_AUTO):
            oracle.set_mode(mode)
            outs.append(oracle.mul_words(a, b))
        oracle.set_mode(MODE_AUTO)
        for o in outs[1:]:
            assert np.array_equal(o, outs[0])
    assert oracle.fft_last_max_err() < 0.25


def test_golden_ntt_kat(oracle, golden):
    for rec in golden["ntt"]["nnt"]:
        k = rec["k"]
        x0 = splitmix64_np(rec["input_seed"], 1 << k) % np.uint64(rec["p"])
        f, p, g, w = oracle.ntt(k, x0)
        assert (p, g, w) == (rec["p"], rec["g"], rec["w"])
        assert _words_md5(f.view(np.uint32)) == rec["fwd_md5"]
        inv, _, _, wi = oracle.ntt(k, f, inverse=True)
        assert wi == rec["w_inv"] and np.array_equal(inv, x0)


def test_naive_dft_small(oracle):
    # natural-order DFT definition X_j = sum x_i w^(ij) (NTT.cpp:191-223)
    k = 4
    n = 1 << k
    x = [int(v) for v in splitmix64_np(3, n) % np.uint64(oracle.prime(11))]
    f, p, g, w = oracle.ntt(k, np.array(x, dtype=np.uint64))
    ref = [sum(x[i] * pow(w, i * j, p) for i in range(n)) % p for j in range(n)]
    assert [int(v) for v in f] == ref


def test_oracle_vs_reference_harness(oracle, reference):
    rng = np.random.default_rng(7)
    for _ in range(150):
        na, nb = (int(v) for v in rng.integers(1, 50, 2))
        a = rng.integers(0, 2 ** 32, na, dtype=np.uint64).astype(np.uint32)
        b = rng.integers(0, 2 ** 32, nb, dtype=np.uint64).astype(np.uint32)
        a[-1] |= 1
        b[-1] |= 1
        A = BF(bool(rng.integers(2)), int(rng.integers(-4, 4)), a)
        B = BF(bool(rng.integers(2)), int(rng.integers(-4, 4)), b)
        p = int(rng.integers(0, 30))
        for name in ("add", "sub", "mul"):
            assert getattr(oracle, name)(A, B, p).same(getattr(reference, name)(A, B, p)), name
        assert oracle.rcp(A, p).same(reference.rcp(A, p))
        assert oracle.ucmp(A, B) == reference.ucmp(A, B)


def test_fft_convention_vs_reference(oracle, reference):
    k = 8
    rng = np.random.default_rng(3)
    x = rng.standard_normal(2 << k)
    for inv in (False, True):
        a = oracle.fft(k, x, inverse=inv)
        b = reference.fft(k, x, inverse=inv)
        assert np.allclose(a, b, rtol=1e-12, atol=1e-9)


# ---- decimal output (BigFloat::to_string_dec, BigFloat.cpp:83-94) -------------

def _dec_case_words(rec):
    w = random_words(rec["seed"], rec["L"])
    if rec["top_mod7"]:
        w[-1] = (w[-1] % 7) + 1
    return w


_DEC_EDGE = {"ones": np.full(300, 0xFFFFFFFF, dtype=np.uint32),
             "zeros_below_top": np.array([0] * 299 + [3], dtype=np.uint32),
             "single_low_bit": np.array([1] + [0] * 298 + [3], dtype=np.uint32)}


def _dec_closed_form(x: BF, digits: int) -> bytes:
    """The closed form the GPU decimal conversion computes: the digits after
    the point are those of N = floor(M 10^D / 2^B), M the words below the top,
    B = 32 (L - 1), D = 9 ceil(digits / 9), written with D digits."""
    import sys
    if hasattr(sys, "set_int_max_str_digits"):
        sys.set_int_max_str_digits(0)  # the decimal text of N has D digits
    w = np.ascontiguousarray(x.words[:-1], dtype="<u4")
    M, B = int.from_bytes(w.tobytes(), "little"), 32 * (x.L - 1)
    D = 9 * ((digits + 8) // 9)
    text = str(int(x.words[-1])) + "." + str((M * 10 ** D) >> B).zfill(D)
    return text[: 2 + digits].encode()


@pytest.mark.parametrize("form", ["literal", "closed"])
def test_decimal_text_matches_reference_numbers(golden, form):
    """Seeded numbers (one- and multi-character integer parts, 0..190,000
    digits) and edge cases, against the reference program's own text."""
    from oracle.ffi import to_string_dec
    conv = to_string_dec if form == "literal" else _dec_closed_form
    for rec in golden["dec"]["numbers"]:
        if form == "literal" and rec["digits"] > 30_000:
            continue  # the nine-digit loop is quadratic; the closed form covers these
        text = conv(BF(True, -rec["L"] + 1, _dec_case_words(rec)), rec["digits"])
        assert len(text) == rec["len"], rec
        if "text" in rec:
            assert text.decode() == rec["text"], rec
        assert hashlib.md5(text).hexdigest() == rec["md5"], rec
    for rec in golden["dec"]["edge"]:
        text = conv(BF(True, 0, _DEC_EDGE[rec["kind"]]), rec["digits"])
        assert hashlib.md5(text).hexdigest() == rec["md5"] and text[-60:].decode() == rec["tail"], rec["kind"]


@pytest.mark.parametrize("digits", [10_000, 100_000])
def test_pi_decimal_text_matches_reference(oracle, golden, digits):
    """Pi()'s final number from the restated operations: its hex text is the
    oracle's pi.txt, and its decimal text (nine-digit loop and closed form)
    is the reference program's to_string_dec of the same number."""
    from oracle.ffi import to_string_dec, to_string_hex
    x = oracle.pi_number(digits)
    hexd, _, _ = oracle.pi_sizes(digits)
    assert to_string_hex(x, hexd) == oracle.pi_hex(digits)
    g = golden["dec"]["pi"][str(digits)]
    lit = to_string_dec(x, digits)
    assert lit == _dec_closed_form(x, digits)
    assert len(lit) == g["len"] and lit[:80].decode() == g["head"] and lit[-80:].decode() == g["tail"]
    assert hashlib.md5(lit).hexdigest() == g["md5"]
