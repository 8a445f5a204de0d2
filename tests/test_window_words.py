"""The window reload of the packed banded-SW sweep (csrc/bsw16.cuh: bsw16_window_words),
restated on the CPU: a lane's two runs of window bytes (its low-half cells g*K + k and
high-half cells H + g*K + k, counted from the row start js - 1) are read with aligned
4-byte loads and funnel shifts instead of one byte load per cell. For every packed
launch shape, lane, window length and row start this checks that

* every cell inside the window gets its window byte, in the register layout the sweep
  uses (word j = bytes of cells 2j lo, 2j hi, 2j+1 lo, 2j+1 hi);
* no load starts past the aligned word that holds the window's last byte, and none
  starts before the aligned word that holds its first byte (each load stays inside
  the 4-byte-aligned span of the window's own bytes).
"""
import random

import pytest

from test_trace_layout import PACKED_SHAPES

M = 0xFFFFFFFF


def prmt(a, b, sel):
    both = (a & M) | ((b & M) << 32)
    out = 0
    for k in range(4):
        n = (sel >> (4 * k)) & 0xF
        out |= ((both >> (8 * (n & 7))) & 0xFF) << (8 * k)
    return out


def funnel_r(lo, hi, s):
    return (((hi << 32) | lo) >> s) & M


def window_words(mem, base, a, b, last, K):
    """bsw16_window_words over byte memory `mem` (addresses relative to `base` = 0):
    returns the words and every address loaded."""
    NW, NU = (K + 1) // 2, (K + 3) // 4
    la = last & ~3
    loads = []

    def at(x):
        x = x if x < la else la
        loads.append(x)
        return int.from_bytes(bytes(mem[x:x + 4]), "little")

    a0, b0 = a & ~3, b & ~3
    sa, sb = (a & 3) * 8, (b & 3) * 8
    wa, wv = at(a0), at(b0)
    wb = [0] * NW
    for m in range(NU):
        na, nb = at(a0 + 4 * (m + 1)), at(b0 + 4 * (m + 1))
        ua, ub = funnel_r(wa, na, sa), funnel_r(wv, nb, sb)
        wb[2 * m] = prmt(ua, ub, 0x5140)
        if 2 * m + 1 < NW:
            wb[2 * m + 1] = prmt(ua, ub, 0x7362)
        wa, wv = na, nb
    return wb, loads


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
def test_window_bytes_and_load_bounds(g, k):
    rng = random.Random(0xB16 + 97 * g + k)
    H = g * k
    for _ in range(60):
        wl = rng.randint(1, 2 * H + 40)
        off = rng.randint(0, 7)             # window start inside its arena
        arena = bytearray(rng.getrandbits(8) for _ in range(off + wl + 16))
        wn = off
        js = rng.randint(1, wl)             # row start column (1-based), js <= wl
        wrow = wn + js - 1
        for gi in range(g):
            c0 = gi * k
            wb, loads = window_words(arena, 0, wrow + c0, wrow + H + c0, wn + wl - 1, k)
            for x in loads:
                assert (wn & ~3) <= x <= ((wn + wl - 1) & ~3), (x, wn, wl)
            for kk in range(k):
                for half, cell in ((0, c0 + kk), (1, H + c0 + kk)):
                    col = js - 1 + cell          # 0-based window column of the cell
                    if col >= wl:
                        continue                 # past the window end: never active
                    j, odd = kk >> 1, kk & 1
                    got = (wb[j] >> (8 * (2 * odd + half))) & 0xFF
                    assert got == arena[wn + col], (g, k, gi, kk, half, js, wl)
