"""Seeded parity corpora shared by the GPU tests (CPU side: inputs + oracle answers)."""
import numpy as np

import pyoracle as O
from refgen import BASES, XorShift

NEXT = {ord("A"): ord("C"), ord("C"): ord("G"), ord("G"): ord("T"), ord("T"): ord("A")}


def mutate(rng, seq: bytes, subs: int, indels: int) -> bytes:
    s = bytearray(seq)
    for _ in range(subs):
        if s:
            p = rng.next() % len(s)
            s[p] = NEXT.get(s[p], ord("A"))
    for _ in range(indels):
        if len(s) < 4:
            break
        p = rng.next() % len(s)
        ln = 1 + rng.next() % 3
        if rng.next() % 2:
            s[p:p] = bytes(BASES[rng.next() % 4] for _ in range(ln))
        else:
            del s[p:p + ln]
    return bytes(s)


def sw_corpus(seed: int, n: int, qmin=20, qmax=200, pad=60, alpha=b"ACGT", max_band=48):
    """(read, window, offset, band, abort) cases around a planted locus."""
    rng = XorShift(seed)
    out = []
    for _ in range(n):
        q = qmin + rng.next() % (qmax - qmin + 1)
        w = q + rng.next() % (pad + 1)
        win = bytes(alpha[rng.next() % len(alpha)] for _ in range(w))
        start = rng.next() % max(1, w - q + 1)
        read = mutate(rng, win[start:start + q], rng.next() % 6, rng.next() % 3)
        if not read:
            read = b"A"
        if rng.next() % 5 == 0:  # unrelated read
            read = bytes(alpha[rng.next() % len(alpha)] for _ in range(len(read)))
        kind = rng.next() % 4
        offset = start if kind else int(rng.next() % (w + 20)) - 10
        band = 1 + rng.next() % max_band
        abort = O.ABORT_DISABLED if rng.next() % 3 else int(rng.next() % (q + 5))
        out.append((read, win, offset, band, abort))
    return out


def oracle_sw(cases, cfg, adaptive=True, max_drift=16, dp_xdrop=None, per_pair_band=True):
    res = []
    for read, win, off, band, abort in cases:
        c = O.OrcCfg(cfg.match_score, cfg.mismatch, cfg.gap_open, cfg.gap_extend,
                     band if per_pair_band else cfg.bandwidth, cfg.xdrop, cfg.clip_penalty)
        res.append(O.banded_sw(read, win, off, c, abort_score=abort, adaptive=adaptive,
                               max_drift=max_drift, dp_xdrop=dp_xdrop))
    return res
