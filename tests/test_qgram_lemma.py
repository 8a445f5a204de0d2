"""The 4-gram prefilter's bound, restated on the CPU: whenever the filter would
reject a (read, window) pair, the oracle's Myers answers None. Small seeded
cases around the threshold (planted reads with edits near k, random windows,
non-ACGT bytes)."""
import pytest

import pyoracle as O
from gpu_cases import mutate
from refgen import XorShift

VALID = {ord(c): i for i, c in enumerate("ACGT")} | {ord(c): i for i, c in enumerate("acgt")}


def grams(seq: bytes):
    """(position, code) of every 4-gram made only of ACGT/acgt bases."""
    out = []
    for p in range(len(seq) - 3):
        w = seq[p:p + 4]
        if all(b in VALID for b in w):
            code = 0
            for b in w:
                code = code * 4 + VALID[b]
            out.append((p, code))
    return out


def qgram_reject(read: bytes, win: bytes, k: int) -> bool:
    need = len(read) - 3 - 4 * k
    if need <= 0 or len(win) < 4:
        return False
    present = {c for _, c in grams(win)}
    return sum(1 for _, c in grams(read) if c in present) < need


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_filter_rejects_only_myers_none(seed):
    rng = XorShift(0xC0FFEE + seed)
    alpha = b"ACGT" if seed < 3 else b"ACGTNacgt"
    rejected = 0
    for _ in range(600):
        m = 20 + rng.next() % 120
        n = m + rng.next() % 120
        win = bytes(alpha[rng.next() % len(alpha)] for _ in range(n))
        k = rng.next() % 12
        start = rng.next() % (n - m + 1)
        if rng.next() % 3:
            read = mutate(rng, win[start:start + m], rng.next() % (k + 4), rng.next() % 4)
        else:
            read = bytes(alpha[rng.next() % len(alpha)] for _ in range(m))
        if not read:
            continue
        if qgram_reject(read, win, k):
            rejected += 1
            assert O.bounded_edit_distance(read, win, k) is None, (read, win, k)
    assert rejected > 50


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_certified_pairs_meet_the_certificate_bound(seed):
    # The filter-first verification skips the sieve of a pair whose 4-gram count is
    # below m - 3 - 4 min(threshold, 2) (the certificate accepts at most two
    # mismatches at its shift, each touching at most four read 4-grams). No pair
    # the oracle certifies may fall below that bound. Planted reads with 0-3
    # substitutions around the certificate's limit; mixed-case bases in one seed (an
    # N only stops the certificate, so it cannot break the bound); thresholds from
    # the router default up to 12.
    rng = XorShift(0xCE27 + seed)
    alpha = b"ACGT" if seed < 3 else b"ACGTACGTacgt"
    certified = 0
    for _ in range(500):
        m = 40 + rng.next() % 110
        n = m + rng.next() % 100
        win = bytes(alpha[rng.next() % len(alpha)] for _ in range(n))
        start = rng.next() % (n - m + 1)
        read = mutate(rng, win[start:start + m], rng.next() % 4, 0)
        thr = (-1, 1, 2, 3, 12)[rng.next() % 5]
        out, _ = O.verify_pair(read, win, O.verify_params(O.cfg(), thr, 8))
        if out.status != 1:
            continue
        certified += 1
        t = O.spectral_max_mismatches(len(read)) if thr < 0 else thr
        present = {c for _, c in grams(win)}
        count = sum(1 for _, c in grams(read) if c in present)
        assert count >= len(read) - 3 - 4 * min(t, 2), (read, win, thr)
    assert certified > 40
