"""The row maximum and its first cell in the packed banded-SW sweep (csrc/bsw16.cuh:
the row-max keys of bsw16_group_sweep), restated on the CPU. Per lane, each half of
word k becomes the key (h << KB) | (2^KB - 1 - k) (one multiply-add on the packed word),
the three-input unsigned 16x2 maxima reduce the words (in two running maxima), the
low half wins ties against the high half, and across lanes the key (h << 11) |
(2047 - cell) is reduced by maximum. The result must be the row's maximum H and the
lowest cell holding it (banded_sw_with keeps the first cell whose H exceeds the running
row maximum, src/alignment/mod.rs:1525-1528),
for every packed shape, whenever every biased H stays below 2^(16 - KB) (the host's
packed_fits bound)."""
import random

import pytest

from test_trace_layout import PACKED_SHAPES


def key_bits(k):
    return 1 if k <= 2 else 2 if k <= 4 else 3 if k <= 8 else 4 if k <= 16 else 5 if k <= 32 else 6


def vimax3_u16x2(a, b, c):
    lo = max(a & 0xFFFF, b & 0xFFFF, c & 0xFFFF)
    hi = max(a >> 16, b >> 16, c >> 16)
    return lo | (hi << 16)


def device_argmax(ph, G, K):
    """ph[g][k] = (lo, hi) biased H of cells g*K + k and H + g*K + k."""
    KB = key_bits(K)
    KM = (1 << KB) - 1
    H = G * K
    best = 0
    for g in range(G):
        c0 = g * K
        mx = mx1 = 0
        for k in range(0, K, 2):
            w = ph[g][k][0] | (ph[g][k][1] << 16)
            ka = (w * (1 << KB) + (KM - k) * 0x10001) & 0xFFFFFFFF
            if k + 1 < K:
                w1 = ph[g][k + 1][0] | (ph[g][k + 1][1] << 16)
                kb = (w1 * (1 << KB) + (KM - (k + 1)) * 0x10001) & 0xFFFFFFFF
            else:
                kb = 0
            if k & 2:
                mx1 = vimax3_u16x2(mx1, ka, kb)
            else:
                mx = vimax3_u16x2(mx, ka, kb)
        mx = vimax3_u16x2(mx, mx1, 0)
        vlo, vhi = (mx & 0xFFFF) >> KB, mx >> (16 + KB)
        lo_first = vlo >= vhi
        idx = c0 + (KM - (mx & KM)) if lo_first else H + c0 + (KM - ((mx >> 16) & KM))
        key = ((vlo if lo_first else vhi) << 11) | (2047 - idx)
        best = max(best, key)
    return best >> 11, 2047 - (best & 2047)


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
def test_row_max_and_first_cell(g, k):
    rng = random.Random(0xA26 + 13 * g + k)
    KB = key_bits(k)
    top = (1 << (16 - KB)) - 1  # packed_fits keeps every biased H at or below this
    H = g * k
    for _ in range(300):
        lo_v = rng.randint(0, top)
        span = rng.choice([1, 2, 4, 16, top - lo_v + 1])
        cells = [min(top, lo_v + rng.randrange(span)) for _ in range(2 * H)]
        ph = [[(cells[gi * k + kk], cells[H + gi * k + kk]) for kk in range(k)] for gi in range(g)]
        m = max(cells)
        assert device_argmax(ph, g, k) == (m, cells.index(m)), (g, k)
