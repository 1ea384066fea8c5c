"""NTT.h / FFT.h drop-ins on the GPU vs the oracle and the reference goldens."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle.ffi import splitmix64_np, random_words

pytestmark = pytest.mark.gpu


def _dev(torch, arr):
    t = torch.from_numpy(np.ascontiguousarray(arr).view(np.int64) if arr.dtype == np.uint64 else
                         np.ascontiguousarray(arr)).cuda()
    return t


def _u64(t):
    return t.cpu().numpy().view(np.uint64)


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 11, 12, 13, 14, 16, 18])
def test_ntt_forward_inverse_vs_oracle(pic, torch_cuda, oracle, k):
    torch = torch_cuda
    n = 1 << k
    p = oracle.prime(max(k, 11))
    x = splitmix64_np(100 + k, n) % np.uint64(p)
    want, wp, _, _ = oracle.ntt(k, x)
    assert wp == p
    t = _dev(torch, x.astype(np.uint64))
    pic.check(pic.lib().pic_ntt_forward(t.data_ptr(), k, _stream(torch)))
    torch.cuda.synchronize()
    got = _u64(t)
    assert np.array_equal(got, want)
    pic.check(pic.lib().pic_ntt_inverse(t.data_ptr(), k, _stream(torch)))
    torch.cuda.synchronize()
    assert np.array_equal(_u64(t), x)


def test_ntt_golden_kat(pic, torch_cuda, golden):
    torch = torch_cuda
    for rec in golden["ntt"]["nnt"]:
        k = rec["k"]
        x0 = splitmix64_np(rec["input_seed"], 1 << k) % np.uint64(rec["p"])
        t = _dev(torch, x0)
        pic.check(pic.lib().pic_ntt_forward(t.data_ptr(), k, _stream(torch)))
        torch.cuda.synchronize()
        f = _u64(t)
        assert hashlib.md5(f.view(np.uint32).astype("<u4").tobytes()).hexdigest() == rec["fwd_md5"]


@pytest.mark.parametrize("k", [22, 24])
def test_ntt_large_roundtrip_and_convolution(pic, torch_cuda, k):
    """Size-independent properties at lengths the oracle is too slow for:
    inverse(forward(x)) == x, and forward is linear."""
    torch = torch_cuda
    n = 1 << k
    p = pic.lib().pic_ntt_prime(k)
    x = splitmix64_np(5, n) % np.uint64(p)
    y = splitmix64_np(6, n) % np.uint64(p)
    tx, ty = _dev(torch, x), _dev(torch, y)
    s = _stream(torch)
    pic.check(pic.lib().pic_ntt_forward(tx.data_ptr(), k, s))
    pic.check(pic.lib().pic_ntt_forward(ty.data_ptr(), k, s))
    xy = (x.astype(object) + y.astype(object)) % p
    txy = _dev(torch, np.array(xy, dtype=np.uint64))
    pic.check(pic.lib().pic_ntt_forward(txy.data_ptr(), k, s))
    torch.cuda.synchronize()
    fx, fy, fxy = _u64(tx), _u64(ty), _u64(txy)
    idx = np.arange(0, n, 9973)
    assert all((int(fx[i]) + int(fy[i])) % p == int(fxy[i]) for i in idx)
    pic.check(pic.lib().pic_ntt_inverse(tx.data_ptr(), k, s))
    torch.cuda.synchronize()
    assert np.array_equal(_u64(tx), x)


def test_int_to_ntt_and_back(pic, torch_cuda, oracle):
    torch = torch_cuda
    k = 12
    a = random_words(9, 700)
    b = random_words(10, 900)
    ta, tb = _dev(torch, a), _dev(torch, b)
    Ta = torch.zeros(1 << k, dtype=torch.int64, device="cuda")
    Tb = torch.zeros(1 << k, dtype=torch.int64, device="cuda")
    L, s = pic.lib(), _stream(torch)
    pic.check(L.pic_int_to_ntt(Ta.data_ptr(), k, ta.data_ptr(), a.size, s))
    pic.check(L.pic_int_to_ntt(Tb.data_ptr(), k, tb.data_ptr(), b.size, s))
    pic.check(L.pic_ntt_forward(Ta.data_ptr(), k, s))
    pic.check(L.pic_ntt_forward(Tb.data_ptr(), k, s))
    pic.check(L.pic_ntt_pointwise(Ta.data_ptr(), Tb.data_ptr(), k, s))
    pic.check(L.pic_ntt_inverse(Ta.data_ptr(), k, s))
    z = torch.zeros(1600, dtype=torch.int32, device="cuda")
    pic.check(L.pic_ntt_to_int(Ta.data_ptr(), k, z.data_ptr(), 1600, s))
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy().view(np.uint32), oracle.mul_words(a, b))
    # the reference's length check: 2^k >= 2 AL (NTT.cpp:352-353)
    assert L.pic_ntt_to_int(Ta.data_ptr(), k, z.data_ptr(), 2049, s) == pic.ERR_LENGTH


def test_fft_api_product_and_error_log(pic, torch_cuda, oracle):
    torch = torch_cuda
    k = 14
    a = random_words(21, 1000)
    b = random_words(22, 1500)
    ta, tb = _dev(torch, a), _dev(torch, b)
    Fa = torch.zeros(2 << k, dtype=torch.float64, device="cuda")
    Fb = torch.zeros(2 << k, dtype=torch.float64, device="cuda")
    L, s = pic.lib(), _stream(torch)
    pic.check(L.pic_int_to_fft(Fa.data_ptr(), k, ta.data_ptr(), a.size, s))
    pic.check(L.pic_int_to_fft(Fb.data_ptr(), k, tb.data_ptr(), b.size, s))
    pic.check(L.pic_fft_forward(Fa.data_ptr(), k, s))
    pic.check(L.pic_fft_forward(Fb.data_ptr(), k, s))
    pic.check(L.pic_fft_pointwise(Fa.data_ptr(), Fb.data_ptr(), k, s))
    pic.check(L.pic_fft_inverse(Fa.data_ptr(), k, s))
    z = torch.zeros(2500, dtype=torch.int32, device="cuda")
    pic.check(L.pic_fft_to_int(Fa.data_ptr(), k, z.data_ptr(), 2500, s))
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy().view(np.uint32), oracle.mul_words(a, b))
    err = L.pic_fft_last_max_err()
    assert 0.0 <= err < 0.25
    assert L.pic_int_to_fft(Fa.data_ptr(), k, ta.data_ptr(), (1 << k) // 4 + 1, s) == pic.ERR_LENGTH


def test_fft_forward_matches_oracle_convention(pic, torch_cuda, oracle):
    torch = torch_cuda
    k = 15
    rng = np.random.default_rng(4)
    x = rng.standard_normal(2 << k)
    t = torch.from_numpy(x.copy()).cuda()
    pic.check(pic.lib().pic_fft_forward(t.data_ptr(), k, _stream(torch)))
    torch.cuda.synchronize()
    want = oracle.fft(k, x)
    assert np.allclose(t.cpu().numpy(), want, rtol=1e-9, atol=1e-8)


@pytest.mark.parametrize("k", [10, 15])
def test_fft_matches_reference_fft(pic, torch_cuda, reference, k):
    """pic_fft_forward / pic_fft_inverse against the reference's own AVX
    fft_forward / fft_inverse (FFT.cpp:64-463, compiled from its sources):
    same sign convention, bit-reversed order and unscaled inverse, to FP64
    rounding (rtol 1e-9)."""
    torch = torch_cuda
    rng = np.random.default_rng(40 + k)
    x = rng.standard_normal(2 << k)
    L = pic.lib()
    for inv in (False, True):
        t = torch.from_numpy(x.copy()).cuda()
        f = L.pic_fft_inverse if inv else L.pic_fft_forward
        pic.check(f(t.data_ptr(), k, _stream(torch)))
        torch.cuda.synchronize()
        want = reference.fft(k, x, inverse=inv)
        assert np.allclose(t.cpu().numpy(), want, rtol=1e-9, atol=1e-8 * (1 << (k // 2)))
