"""The one-cell realignment of the packed banded-SW sweep (csrc/bsw16.cuh:
bsw16_shift1), restated on the CPU against the general realignment (bsw16_realign:
cell c <- old cell c + s, neutral outside [0, prev_len)). Lane g's word k holds cell
g*K + k in its low half and H + g*K + k in its high half (H = G*K); the previous row's
cells at and beyond its length are already neutral (H = the bias, E = 0), which the
one-cell shifts rely on instead of testing bounds. Checked for s = -1 (the band stayed)
and s = +1 (the band moved two columns), every packed shape and previous row length."""
import random

import pytest

from test_trace_layout import PACKED_SHAPES

BIAS = 0x1234  # any neutral H value


def cell_of(g, k, half, G, K):
    return half * G * K + g * K + k


def general(old, s, prev_len, G, K, neutral):
    """bsw16_realign: per lane / word / half the shifted cell, or neutral."""
    out = {}
    for g in range(G):
        for k in range(K):
            for half in (0, 1):
                src = cell_of(g, k, half, G, K) + s
                out[(g, k, half)] = old[src] if 0 <= src < prev_len else neutral
    return out


def shift1(regs, down, G, K, neutral):
    """bsw16_shift1 over registers regs[g][k] = (lo, hi)."""
    out = {}
    for g in range(G):
        if down:  # cell c <- c - 1: previous lane's word K-1; lane 0: none / last lane's lo
            lo, hi = regs[(g + G - 1) % G][K - 1]
            if g == 0:
                lo, hi = neutral, lo
            new = [(lo, hi)] + [regs[g][k - 1] for k in range(1, K)]
        else:  # cell c <- c + 1: next lane's word 0; last lane: lane 0's hi / none
            lo, hi = regs[(g + 1) % G][0]
            if g == G - 1:
                lo, hi = hi, neutral
            new = [regs[g][k + 1] for k in range(K - 1)] + [(lo, hi)]
        for k in range(K):
            out[(g, k, 0)], out[(g, k, 1)] = new[k]
    return out


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
def test_one_cell_shifts_equal_the_general_realignment(g, k):
    G, K = g, k
    cap = 2 * G * K
    rng = random.Random(0x5E1F + 31 * G + K)
    for prev_len in sorted({1, 2, G * K - 1, G * K, G * K + 1, cap - 1, cap,
                            rng.randint(1, cap), rng.randint(1, cap)}):
        if not 1 <= prev_len <= cap:
            continue
        # the previous row: real values inside its length, neutral beyond (masked)
        old = [rng.randint(0, 0xFFFF) if c < prev_len else BIAS for c in range(cap)]
        regs = [[(old[cell_of(gg, kk, 0, G, K)], old[cell_of(gg, kk, 1, G, K)])
                 for kk in range(K)] for gg in range(G)]
        for s, down in ((-1, True), (1, False)):
            assert shift1(regs, down, G, K, BIAS) == general(old, s, prev_len, G, K, BIAS), \
                (G, K, prev_len, s)
