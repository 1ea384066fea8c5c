"""The binary-splitting slot capacities (bsr.cu, slot_caps) hold every merge
they are used for: checked in exact integer arithmetic on the CPU, beyond
the sizes the GPU tests reach.

A level's P, Q, R slots hold ceil(bound / 32) + 3 words (+ 4 for P), the
bound for a node of n leaves ending at term T being
    log2 Q <= n log2(10939058860032000 (T + 1)^3)      (Q_j = C j^3, j <= T)
    log2 R <= n log2(72 (T + 1)^3)                     ((2j-1)(6j-5)(6j-1) < 72 j^3)
    log2 |P| <= log2 Q + log2(n (0.0895 + 3.6e-6 T) + 1) + 1
(|P| / Q is at most the sum of the leaves' |P_j| / Q_j < 8.95e-8 + 3.59e-6 j).
A merge writes the full product width, na + nb words, and P's carry word, so
the test checks those widths, with the node's own leaf count and last term
(the level's caps use the level's largest node and the last term of the
whole series, which are never smaller).  The nodes at the far end of a range
fill their slots to within a few words: the margins are what keep them in."""
from __future__ import annotations

import math
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _caps(n: int, T: int):
    """slot_caps restated (bsr.cu)."""
    lq = math.log2(10939058860032000.0) + 3.0 * math.log2(T + 1.0)
    lr = math.log2(72.0) + 3.0 * math.log2(T + 1.0)
    bq, br = n * lq, n * lr
    bp = bq + math.log2(n * (0.0895 + 3.6e-6 * T) + 1.0) + 1.0
    return math.ceil(bp / 32.0) + 4, math.ceil(bq / 32.0) + 3, math.ceil(br / 32.0) + 3


def _words(x: int) -> int:
    return (abs(x).bit_length() + 31) // 32


def _node(a: int, b: int, fill: list):
    """P, Q, R of [a, b) by the reference's recursion (PI.h:64-112), checking
    every merge's product widths against the caps."""
    if b - a == 1:
        P = (13591409 + 545140134 * b) * (2 * b - 1) * (6 * b - 5) * (6 * b - 1)
        return (-P if b % 2 else P), 10939058860032000 * b ** 3, (2 * b - 1) * (6 * b - 5) * (6 * b - 1)
    m = (a + b) // 2
    P0, Q0, R0 = _node(a, m, fill)
    P1, Q1, R1 = _node(m, b, fill)
    cP, cQ, cR = _caps(b - a, b)
    need = (max(_words(P0) + _words(Q1), _words(P1) + _words(R0)) + 1, _words(Q0) + _words(Q1),
            _words(R0) + _words(R1))
    assert need[0] <= cP and need[1] <= cQ and need[2] <= cR, (a, b, need, (cP, cQ, cR))
    fill[0] = max(fill[0], need[0] / cP, need[1] / cQ, need[2] / cR)
    return P0 * Q1 + P1 * R0, Q0 * Q1, R0 * R1


def test_slot_caps_restatement_matches_the_source():
    src = open(os.path.join(ROOT, "piculator_b200", "csrc", "bsr.cu")).read()
    for frag in ("log2(10939058860032000.0) + 3.0 * log2(T + 1.0)", "log2(72.0) + 3.0 * log2(T + 1.0)",
                 "log2(n * (0.0895 + 3.6e-6 * T) + 1.0) + 1.0", "ceil(bq / 32.0) + 3", "ceil(br / 32.0) + 3",
                 "ceil(bp / 32.0) + 4"):
        assert frag in src, frag


def test_every_merge_of_a_whole_small_series_fits():
    fill = [0.0]
    _node(0, 3000, fill)
    assert fill[0] <= 1.0


# the last terms of the series at 1e9 and 3e9 digits, and near the 2^32 limit
@pytest.mark.parametrize("end,size", [(70_513_670, 4096), (211_541_010, 2048), (4_000_000_000, 1024)])
def test_merges_at_the_far_end_of_large_series_fit(end, size):
    fill = [0.0]
    _node(end - size, end, fill)
    assert fill[0] <= 1.0


def _leaf(b: int):
    P = (13591409 + 545140134 * b) * (2 * b - 1) * (6 * b - 5) * (6 * b - 1)
    return P, 10939058860032000 * b ** 3, (2 * b - 1) * (6 * b - 5) * (6 * b - 1)


def test_bottom_kernel_register_widths_hold_up_to_the_term_limit():
    """The bottom depth's leaves and two-leaf merges are formed in fixed
    register arrays (bsr.cu: LeafV's SW<6> / SW<5> / SW<4>, the merge's
    SW<12> / SW<10> / SW<8>).  The largest values, at the last terms below the
    reference's 2^32-term limit (PI.h:149-151), fit with the carry word."""
    import re
    src = open(os.path.join(ROOT, "piculator_b200", "csrc", "bsr.cu")).read()
    leaf = re.search(r"struct LeafV \{\s*SW<(\d+)> P;\s*bool sP;\s*SW<(\d+)> Q;\s*SW<(\d+)> R;", src)
    merge = re.search(r"SW<(\d+)> t1, t2, P;.*?SW<(\d+)> Q;\s*SW<(\d+)> R;", src, re.S)
    assert leaf and merge
    lp, lq, lr = (32 * int(v) for v in leaf.groups())
    mp, mq, mr = (32 * int(v) for v in merge.groups())
    b = 2 ** 32 - 1
    P0, Q0, R0 = _leaf(b - 1)
    P1, Q1, R1 = _leaf(b)
    assert P1.bit_length() <= lp and Q1.bit_length() <= lq and R1.bit_length() <= lr
    # P0 Q1 + P1 R0 with both signs alike (the sum), Q0 Q1, R0 R1
    assert (P0 * Q1 + P1 * R0).bit_length() <= mp
    assert (Q0 * Q1).bit_length() <= mq and (R0 * R1).bit_length() <= mr
