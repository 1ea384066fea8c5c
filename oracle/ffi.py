"""ctypes bindings for the two CPU checkers (test infrastructure only).

* ``Oracle`` loads ``oracle/_build/liboracle.so``, the C restatement of the
  reference's multiply path (``pic_oracle.c``).
* ``Reference`` loads ``oracle/_ref/libpicref.so``, the reference's own
  BigFloat.cpp / FFT.cpp / NTT.cpp compiled in place with ``ref_harness.cpp``.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  Values cross the boundary as ``BF`` tuples
``(sign, exp, words)`` with ``sign`` True for positive/zero and ``words`` a
little-endian ``numpy.uint32`` array, mirroring BigFloat.h:33-36.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import NamedTuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpicref.so")
REF_PI = os.path.join(HERE, "_ref", "picref_pi")

OP_MUL, OP_ADD, OP_SUB, OP_MUL_U32, OP_RCP, OP_DIV, OP_INVSQRT, OP_UCMP = range(8)
MODE_AUTO, MODE_SCHOOL, MODE_FFT, MODE_NTT = range(4)


class BF(NamedTuple):
    sign: bool
    exp: int
    words: np.ndarray  # uint32

    @property
    def L(self) -> int:
        return int(self.words.size)

    def to_int(self) -> int:
        """Signed integer value of the mantissa (exponent not applied)."""
        v = int.from_bytes(self.words.astype("<u4").tobytes(), "little")
        return v if self.sign else -v

    @staticmethod
    def from_int(v: int, exp: int = 0) -> "BF":
        sign = v >= 0
        v = abs(v)
        n = (v.bit_length() + 31) // 32
        w = np.frombuffer(v.to_bytes(4 * n, "little"), dtype="<u4").astype(np.uint32)
        return BF(sign, exp, w)

    def same(self, other: "BF") -> bool:
        return (self.sign == other.sign and self.exp == other.exp
                and self.L == other.L and bool(np.array_equal(self.words, other.words)))


class _CBF(C.Structure):
    _fields_ = [("sign", C.c_int32), ("exp", C.c_int64), ("L", C.c_uint64),
                ("T", C.POINTER(C.c_uint32))]


def _to_c(x: BF | None):
    if x is None:
        return None, None
    w = np.ascontiguousarray(x.words, dtype=np.uint32)
    c = _CBF(1 if x.sign else 0, int(x.exp), int(w.size),
             w.ctypes.data_as(C.POINTER(C.c_uint32)))
    return c, w


class _Lib:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run make -C oracle)")
        self.lib = C.CDLL(path)
        f = getattr(self.lib, self.prefix + "bf_op")
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.POINTER(_CBF), C.POINTER(_CBF), C.c_uint64, C.c_uint64,
                      C.c_int, C.POINTER(_CBF), C.c_uint64] if self.prefix == "ref_" else \
            [C.c_int, C.POINTER(_CBF), C.POINTER(_CBF), C.c_uint64, C.c_uint64,
             C.POINTER(_CBF), C.c_uint64]
        self._op = f

    def _call(self, op, a, b, p, s, cap, threads):
        ca, wa = _to_c(a)
        cb, wb = _to_c(b)
        while True:
            out = np.zeros(max(cap, 1), dtype=np.uint32)
            co = _CBF(0, 0, 0, out.ctypes.data_as(C.POINTER(C.c_uint32)))
            pa = C.byref(ca) if ca is not None else None
            pb = C.byref(cb) if cb is not None else None
            if self.prefix == "ref_":
                rc = self._op(op, pa, pb, p, s, threads, C.byref(co), cap)
            else:
                rc = self._op(op, pa, pb, p, s, C.byref(co), cap)
            if op == OP_UCMP:
                return rc - 10
            if rc == -1:
                cap = int(co.L) + 1
                continue
            if rc == -2:
                raise ZeroDivisionError("reference throws: Divide by Zero")
            if rc != 0:
                raise RuntimeError(f"bf_op failed rc={rc}")
            return BF(bool(co.sign), int(co.exp), out[: int(co.L)].copy())

    def _cap(self, a, b):
        la = a.L if a is not None else 0
        lb = b.L if b is not None else 0
        return la + lb + 8

    def mul(self, a, b, p=0, threads=1):
        return self._call(OP_MUL, a, b, p, 0, self._cap(a, b), threads)

    def add(self, a, b, p=0):
        return self._call(OP_ADD, a, b, p, 0, self._cap(a, b), 1)

    def sub(self, a, b, p=0):
        return self._call(OP_SUB, a, b, p, 0, self._cap(a, b), 1)

    def mul_u32(self, a, s):
        return self._call(OP_MUL_U32, a, None, 0, s, self._cap(a, None), 1)

    def rcp(self, a, p, threads=1):
        return self._call(OP_RCP, a, None, p, 0, p + 8, threads)

    def div(self, a, b, p, threads=1):
        return self._call(OP_DIV, a, b, p, 0, 2 * p + 8, threads)

    def invsqrt(self, x, p, threads=1):
        return self._call(OP_INVSQRT, None, None, p, x, 2 * p + 8, threads)

    def ucmp(self, a, b):
        return self._call(OP_UCMP, a, b, 0, 0, 1, 1)


class Oracle(_Lib):
    """The C restatement (pic_oracle.c)."""
    prefix = "oracle_"

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.oracle_set_mode.argtypes = [C.c_int]
        L.oracle_get_mode.restype = C.c_int
        L.oracle_mul_words.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]
        L.oracle_ntt.argtypes = [C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.oracle_fft.argtypes = [C.c_int, C.c_int, C.c_void_p]
        L.oracle_fft_last_max_err.restype = C.c_double
        L.oracle_fft_recomputes.restype = C.c_uint64
        L.oracle_prime.argtypes = [C.c_int]
        L.oracle_prime.restype = C.c_uint64
        L.oracle_generator.argtypes = [C.c_uint64]
        L.oracle_generator.restype = C.c_uint64
        L.oracle_bsr.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(_CBF),
                                 C.POINTER(_CBF), C.POINTER(_CBF), C.c_uint64]
        L.oracle_pi_hex.argtypes = [C.c_uint64, C.c_char_p, C.c_uint64]
        L.oracle_pi_hex.restype = C.c_int64
        L.oracle_pi_sizes.argtypes = [C.c_uint64] + [C.POINTER(C.c_uint64)] * 3

    def set_mode(self, mode: int):
        self.lib.oracle_set_mode(mode)

    def mul_words(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        z = np.zeros(a.size + b.size, dtype=np.uint32)
        self.lib.oracle_mul_words(a.ctypes.data, a.size, b.ctypes.data, b.size, z.ctypes.data)
        return z

    def ntt(self, k: int, data: np.ndarray, inverse: bool = False):
        d = np.ascontiguousarray(data, dtype=np.uint64).copy()
        p, g, w = C.c_uint64(), C.c_uint64(), C.c_uint64()
        rc = self.lib.oracle_ntt(k, int(inverse), d.ctypes.data, C.byref(p), C.byref(g), C.byref(w))
        if rc:
            raise ValueError(k)
        return d, int(p.value), int(g.value), int(w.value)

    def fft(self, k: int, data: np.ndarray, inverse: bool = False) -> np.ndarray:
        d = np.ascontiguousarray(data, dtype=np.float64).copy()
        self.lib.oracle_fft(k, int(inverse), d.ctypes.data)
        return d

    def fft_last_max_err(self) -> float:
        return float(self.lib.oracle_fft_last_max_err())

    def fft_recomputes(self) -> int:
        return int(self.lib.oracle_fft_recomputes())

    def prime(self, k: int) -> int:
        return int(self.lib.oracle_prime(k))

    def generator(self, p: int) -> int:
        return int(self.lib.oracle_generator(p))

    def bsr(self, a: int, b: int, p: int):
        cap = 64 + 8 * (b - a)
        while True:
            bufs = [np.zeros(cap, dtype=np.uint32) for _ in range(3)]
            cs = [_CBF(0, 0, 0, x.ctypes.data_as(C.POINTER(C.c_uint32))) for x in bufs]
            rc = self.lib.oracle_bsr(a, b, p, C.byref(cs[0]), C.byref(cs[1]), C.byref(cs[2]), cap)
            if rc == -1:
                cap *= 4
                continue
            if rc:
                raise RuntimeError(rc)
            return tuple(BF(bool(c.sign), int(c.exp), x[: int(c.L)].copy()) for c, x in zip(cs, bufs))

    def pi_sizes(self, digits: int):
        h, p, t = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.lib.oracle_pi_sizes(digits, C.byref(h), C.byref(p), C.byref(t))
        return int(h.value), int(p.value), int(t.value)

    def pi_hex(self, digits: int) -> bytes:
        hexd, _, _ = self.pi_sizes(digits)
        cap = hexd + 64
        buf = C.create_string_buffer(cap)
        n = self.lib.oracle_pi_hex(digits, buf, cap)
        if n < 0:
            raise RuntimeError(n)
        return buf.raw[:n]

    def pi_number(self, digits: int) -> BF:
        """Pi()'s final number before base conversion (PI.h:176-199), composed
        from the restated operations: the series, the combination with
        13591409 and 4270934400, the division, invsqrt(10005) and the final
        product, each at precision p."""
        _, p, terms = self.pi_sizes(digits)
        P, Q, _ = self.bsr(0, terms, p)
        P = self.add(self.mul_u32(Q, 13591409), P, p)
        Q = self.mul_u32(Q, 4270934400)
        P = self.div(Q, P, p)
        return self.mul(P, self.invsqrt(10005, p), p)


def _below_top(x: BF) -> tuple[int, int]:
    """(M, B): the integer held by every word below the top one, and its bit
    width B = 32 (L - 1)."""
    w = np.ascontiguousarray(x.words[:-1], dtype="<u4")
    return int.from_bytes(w.tobytes(), "little"), 32 * (x.L - 1)


def to_string_dec(x: BF, digits: int) -> bytes:
    """BigFloat::to_string_dec (BigFloat.cpp:83-94): the top word in decimal,
    a point, then nine digits per round -- clear the top word, multiply the
    number by 10^9 (mul(uint32), BigFloat.cpp:156-183) and print the new top
    word -- and the text cut to 2 + digits characters.  With the top word
    cleared the multiply never carries out of the top word, so the length
    stays L and each round is M <- M 10^9, digit group = M >> B, M <- M mod
    2^B on the words below the top.  Sign and exponent are not printed."""
    M, B = _below_top(x)
    mask = (1 << B) - 1
    out = [str(int(x.words[-1])), "."]
    for _ in range((digits + 8) // 9):
        M *= 1_000_000_000
        out.append("%09d" % (M >> B))
        M &= mask
    return "".join(out)[: 2 + digits].encode()


def to_string_hex(x: BF, digits: int) -> bytes:
    """BigFloat::to_string_hex (BigFloat.cpp:95-106): the top word in decimal,
    a point, then the words below it from the top down as eight hex digits
    each, cut to 2 + digits characters."""
    w = x.words
    if (digits + 7) // 8 > x.L - 1:
        raise ValueError("more hex digits than words below the top (the reference reads before T[0])")
    groups = "".join("%08x" % int(w[x.L - 2 - i]) for i in range((digits + 7) // 8))
    return (str(int(w[-1])) + "." + groups)[: 2 + digits].encode()


class Reference(_Lib):
    """The reference's own code (oracle/_ref/libpicref.so)."""
    prefix = "ref_"

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        L.ref_nnt.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_uint64),
                              C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.ref_fft.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int]
        L.ref_bf_to_hex.argtypes = [C.POINTER(_CBF), C.c_uint64, C.c_char_p, C.c_uint64]
        for n in ("ref_int_to_fft", "ref_fft_to_int", "ref_int_to_ntt", "ref_ntt_to_int"):
            getattr(L, n).argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_uint64]

    def ntt(self, k: int, data: np.ndarray, inverse: bool = False, threads: int = 1):
        d = np.ascontiguousarray(data, dtype=np.uint64).copy()
        p, g, w = C.c_uint64(), C.c_uint64(), C.c_uint64()
        rc = self.lib.ref_nnt(k, int(inverse), d.ctypes.data, threads, C.byref(p), C.byref(g),
                              C.byref(w))
        if rc:
            raise ValueError(k)
        return d, int(p.value), int(g.value), int(w.value)

    def fft(self, k: int, data: np.ndarray, inverse: bool = False, threads: int = 1):
        d = np.ascontiguousarray(data, dtype=np.float64).copy()
        self.lib.ref_fft(k, int(inverse), d.ctypes.data, threads)
        return d

    def to_hex(self, x: BF, digits: int) -> bytes:
        c, w = _to_c(x)
        buf = C.create_string_buffer(digits + 64)
        rc = self.lib.ref_bf_to_hex(C.byref(c), digits, buf, digits + 64)
        if rc:
            raise RuntimeError(rc)
        return buf.value


def splitmix64(seed: int, n: int) -> np.ndarray:
    """splitmix64 stream (Steele, Lea, Flood 2014) as uint64 -- the seeded
    generator for synthetic operands."""
    out = np.empty(n, dtype=np.uint64)
    x = seed & 0xFFFFFFFFFFFFFFFF
    M = 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        x = (x + 0x9E3779B97F4A7C15) & M
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        out[i] = z ^ (z >> 31)
    return out


def splitmix64_np(seed: int, n: int) -> np.ndarray:
    """Vectorised splitmix64: element i is the (i+1)-th output of the stream."""
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        x = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def random_words(seed: int, n: int) -> np.ndarray:
    """n uniform 32-bit limbs: the low halves of a splitmix64 stream."""
    return (splitmix64_np(seed, n) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
