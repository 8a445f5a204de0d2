"""The per-word activity masks of the packed banded-SW sweep (csrc/bsw16.cuh:
bsw16_act), restated on the CPU. Every row now runs the masked form, so every word of
every row takes its mask from d0 = D0B + (row_len, row_len) with D0B = (2^15 - 1 - c0,
2^15 - 1 - H - c0) per half (c0 = g*K): word k's mask is PRMT 0xBB99 of d0 - k*0x10001,
which replicates bit 15 of each half. It must be 0xFFFF exactly for the halves whose
cell (g*K + k low, H + g*K + k high) lies inside the row, for every packed shape, lane
and row length from 0 to the row capacity, with no borrow between the halves."""
import pytest

from test_trace_layout import PACKED_SHAPES

M = 0xFFFFFFFF


def isum(lo, hi):
    return ((hi & 0xFFFF) * 65536 + (lo & 0xFFFF)) & M


def prmt_bb99(x):
    b1, b3 = (x >> 8) & 0xFF, (x >> 24) & 0xFF
    lo = 0xFFFF if b1 & 0x80 else 0
    hi = 0xFFFF if b3 & 0x80 else 0
    return lo | (hi << 16)


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
def test_masks_mark_the_cells_inside_the_row(g, k):
    H = g * k
    for gi in range(g):
        c0 = gi * k
        d0b = isum(0x8000 - 1 - c0, 0x8000 - 1 - H - c0)
        for row_len in range(0, 2 * H + 1):
            d0 = (d0b + isum(row_len, row_len)) & M
            for kk in range(k):
                x = (d0 - kk * 0x10001) & M
                # no borrow across the halves: each half's own difference stays >= 0
                assert (x & 0xFFFF) == 0x8000 - 1 - c0 + row_len - kk
                want = (0xFFFF if c0 + kk < row_len else 0) | \
                       ((0xFFFF if H + c0 + kk < row_len else 0) << 16)
                assert prmt_bb99(x) == want, (g, k, gi, row_len, kk)
