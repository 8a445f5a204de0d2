"""The packed banded-SW trace stores no STOP direction: a cell with H = 0 carries
the flags of a diagonal move, and the traceback (warp_walk_scored, csrc/bsw16.cuh)
instead carries the value of the cell it stands on and stops where an H-state cell's
value is 0. Restated here cell by cell over the oracle's DP matrix (banded_sw_with,
mod.rs:1370-1650): the carried value equals the matrix's H at every H-state cell,
and the walk gives the oracle's start coordinates and CIGAR on random corpora under
several scoring schemes (gap open 0 included), bands, offsets and abort bounds."""
import ctypes as C

import numpy as np
import pytest

import pyoracle as O
from gpu_cases import sw_corpus

DIR_MASK, STOP, DIAG, E, F = 3, 0, 1, 2, 3


def _matrix(read, win, off, c, abort):
    q = len(read)
    cap = 2 * c.bandwidth + 2
    out = O.OrcSwResult()
    cig = (C.c_uint32 * (q + len(win) + 2))()
    rs = np.zeros(q + 1, np.int32)
    rl = np.zeros(q + 1, np.int32)
    h = np.zeros((q + 1) * cap, np.int32)
    tr = np.zeros((q + 1) * cap, np.uint8)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = O.lib().orc_banded_sw_matrix(read, q, win, len(win), off, C.byref(c), abort, 1, 16,
                                      c.xdrop, C.byref(out), cig, len(cig), p(rs), p(rl), p(h),
                                      p(tr), cap)
    assert rc == 1
    res = O._swres(out, cig)
    return res, rs, rl, h.reshape(q + 1, cap), tr.reshape(q + 1, cap)


def _scored_walk(read, win, res, rs, rl, h, tr, c):
    go, ge = c.gap_open, c.gap_extend
    i, j, v = res.read_end, res.ref_end, res.score
    state, ops = "H", []
    while i > 0 and j > 0:
        idx = j - rs[i]
        if idx < 0 or idx >= rl[i]:
            break
        t = int(tr[i, idx])
        d = t & DIR_MASK
        if d == STOP:  # the packed flags of an H = 0 cell read as a diagonal move
            d = DIAG
        if state == "H":
            assert v == h[i, idx], (i, j, v, h[i, idx])
            if v == 0:
                break
            if d == DIAG:
                ops.append("M")
                v -= c.match_score if read[i - 1] == win[j - 1] else -c.mismatch
                i, j = i - 1, j - 1
            else:
                state = "E" if d == E else "F"
        elif state == "E":
            ops.append("I")
            i -= 1
            if t & 4:
                v += ge
            else:
                v += go + ge
                state = "H"
        else:
            ops.append("D")
            j -= 1
            if t & 8:
                v += ge
            else:
                v += go + ge
                state = "H"
    runs = []
    for o in reversed(ops):
        if runs and runs[-1][1] == o:
            runs[-1][0] += 1
        else:
            runs.append([1, o])
    return i, j, [(n, o) for n, o in runs]


@pytest.mark.parametrize("scheme", [(1, 4, 6, 1), (2, 3, 5, 2), (1, 4, 0, 1), (1, 1, 2, 0)])
def test_scored_walk_equals_stop_walk(scheme):
    m, x, go, ge = scheme
    cases = sw_corpus(0x5C0E + go, 400, qmin=10, qmax=160, pad=60, max_band=40)
    for read, win, off, band, abort in cases:
        c = O.OrcCfg(m, x, go, ge, band, 100, 5)
        res, rs, rl, h, tr = _matrix(read, win, off, c, abort)
        i, j, cig = _scored_walk(read, win, res, rs, rl, h, tr, c)
        assert (i, j) == (res.read_start, res.ref_start)
        want = [(n, o) for n, o in res.cigar]
        assert cig == want, (read, win, off, band)
