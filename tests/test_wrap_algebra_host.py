"""The wrapped-product identity the three-prime products and binary-splitting
merges rely on, checked in exact integer arithmetic on the CPU.

A product of operands of sa and sb pieces has L = sa + sb - 1 coefficients.
When a power of two Nm with sa, sb <= Nm < L is used as the main cyclic
length, the cyclic product holds c_j + c_(Nm + j) for j < W = L - Nm.  The W
top coefficients depend only on the top W pieces of each operand (a from
index Nm - sb + 1, b from Nm - sa + 1); their product d, taken cyclically at
a length T >= 2W - 1, gives c_(Nm + j) = d_(W - 1 + j) with no wrap.  The
fix-up subtracts d_(W - 1 + j) from y_j and stores it at y_(Nm + j), which
must give the linear product exactly (the GPU kernel does this per prime on
residues, with the inverse-transform scales Nm and T matched)."""
from __future__ import annotations

import numpy as np
import pytest


def _cyclic(a, b, n):
    """Exact cyclic convolution of integer sequences at length n."""
    out = [0] * n
    for i, x in enumerate(a):
        if x:
            for j, y in enumerate(b):
                out[(i + j) % n] += x * y
    return out


def _linear(a, b):
    out = [0] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            out[i + j] += x * y
    return out


def _wrapped(a, b, Nm):
    sa, sb = len(a), len(b)
    L = sa + sb - 1
    assert max(sa, sb) <= Nm < L
    W = L - Nm
    T = 1
    while T < 2 * W - 1:
        T *= 2
    y = _cyclic(a, b, Nm) + [0] * W
    at, bt = a[Nm - sb + 1:], b[Nm - sa + 1:]
    assert len(at) == W and len(bt) == W
    d = _cyclic(at, bt, T)
    for j in range(W):
        h = d[W - 1 + j]
        y[j] -= h
        y[Nm + j] = h
    return y, W, T


@pytest.mark.parametrize("seed", range(12))
def test_wrapped_fixup_gives_the_linear_product(seed):
    rng = np.random.default_rng(seed)
    for _ in range(20):
        Nm = 1 << int(rng.integers(2, 7))
        # both operands at most Nm pieces, product longer than Nm
        sa = int(rng.integers(Nm // 2 + 1, Nm + 1))
        sb = int(rng.integers(max(1, Nm + 2 - sa), Nm + 1))
        a = [int(v) for v in rng.integers(0, 2 ** 56, sa, dtype=np.uint64)]
        b = [int(v) for v in rng.integers(0, 2 ** 56, sb, dtype=np.uint64)]
        y, W, T = _wrapped(a, b, Nm)
        assert y == _linear(a, b), (sa, sb, Nm, W, T)


def test_top_coefficients_depend_only_on_the_top_pieces():
    rng = np.random.default_rng(99)
    sa, sb, Nm = 27, 23, 32
    W = sa + sb - 1 - Nm
    a = [int(v) for v in rng.integers(0, 2 ** 32, sa, dtype=np.uint64)]
    b = [int(v) for v in rng.integers(0, 2 ** 32, sb, dtype=np.uint64)]
    top = _linear(a, b)[Nm:]
    # change every piece below the top W of each operand: the top W coefficients stay
    a2 = [int(v) for v in rng.integers(0, 2 ** 32, Nm - sb + 1, dtype=np.uint64)] + a[Nm - sb + 1:]
    b2 = [int(v) for v in rng.integers(0, 2 ** 32, Nm - sa + 1, dtype=np.uint64)] + b[Nm - sa + 1:]
    assert len(top) == W and _linear(a2, b2)[Nm:] == top


def test_edge_single_wrapped_coefficient():
    # L = Nm + 1: one wrapped coefficient, tail length T = 1
    a, b = [3, 5, 7, 11], [13, 17]
    y, W, T = _wrapped(a, b, 4)
    assert (W, T) == (1, 1) and y == _linear(a, b)
