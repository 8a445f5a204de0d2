"""align_batch_simd drop-in on the GPU vs the oracle's align_batch_simd (the AVX2
i16 / AVX-VNNI i8 full-window kernels restated with their intrinsics, and the
scalar banded fallback): every SimdMode, group boundaries at 16 / 32 inputs,
abort bounds (the all-lanes-done break), mixed shapes and the i16 fit check
(tests/alignment.rs:124-274)."""
import pytest

import pyoracle as O
from gpu_cases import mutate
from refgen import BASES, XorShift

pytestmark = pytest.mark.gpu
MODES = [(O.SIMD_AVX2, O.SIMD_AVX2), (O.SIMD_AVX2, O.SIMD_VNNI), (O.SIMD_VNNI, O.SIMD_VNNI),
         (O.SIMD_SCALAR, O.SIMD_VNNI), (O.SIMD_NEON, O.SIMD_VNNI), (O.SIMD_VNNI, O.SIMD_AVX2)]


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _cmp(ctx, reads, wins, c, mode, detected, aborts=None, offsets=None):
    from kira_ls_aligner_b200 import AlignmentConfig, PairBatch, results_to_list
    n = len(reads)
    aborts = aborts if aborts is not None else [O.ABORT_DISABLED] * n
    offsets = offsets if offsets is not None else [0] * n
    want = O.align_batch_simd(reads, wins, c, mode, detected, aborts=aborts, offsets=offsets)
    cfg = AlignmentConfig(c.match_score, c.mismatch, c.gap_open, c.gap_extend, c.bandwidth,
                          c.xdrop, c.clip_penalty, True, 16)
    b = PairBatch.from_pairs(reads, wins, band_offset=offsets, abort_score=aborts)
    res, ops = ctx.align_batch_simd(b, cfg, mode, detected)
    got = results_to_list(res, ops)
    assert len(got) == len(want) == n
    for i, (g, w) in enumerate(zip(got, want)):
        assert g.key() == w.key(), (i, mode, detected, g, w)


def _batch(rng, n, q, r):
    reads, wins = [], []
    for _ in range(n):
        win = bytes(BASES[rng.next() % 4] for _ in range(r))
        s = rng.next() % (r - q + 1)
        read = mutate(rng, win[s:s + q], rng.next() % 6, rng.next() % 2)
        read = (read + bytes(BASES[rng.next() % 4] for _ in range(q)))[:q]
        if rng.next() % 6 == 0:
            read = bytes(BASES[rng.next() % 4] for _ in range(q))
        reads.append(read)
        wins.append(win)
    return reads, wins


@pytest.mark.parametrize("n", [1, 5, 16, 17, 32, 33, 70])
def test_modes_and_group_sizes(ctx, n):
    rng = XorShift(0xA82 + n)
    reads, wins = _batch(rng, n, 100, 180)
    c = O.cfg(1, 4, 6, 1, 33, 100, 5)
    for mode, det in MODES:
        _cmp(ctx, reads, wins, c, mode, det)


def test_abort_groups(ctx):
    # Per-input abort bounds: a group breaks only when every member is done.
    rng = XorShift(0xAB0)
    c = O.cfg(1, 4, 6, 1, 33, 100, 5)
    for trial in range(6):
        n = 1 + rng.next() % 40
        q = 30 + rng.next() % 80
        reads, wins = _batch(rng, n, q, q + 20 + rng.next() % 60)
        aborts = [O.ABORT_DISABLED if rng.next() % 4 == 0 else int(rng.next() % (q + 20))
                  for _ in range(n)]
        for mode, det in MODES:
            _cmp(ctx, reads, wins, c, mode, det, aborts=aborts)


def test_mixed_shapes_and_fit_failure(ctx):
    rng = XorShift(0xF17)
    r1, w1 = _batch(rng, 6, 60, 120)
    r2, w2 = _batch(rng, 5, 59, 120)
    c = O.cfg(2, 4, 6, 1, 12, 40, 5)
    offs = [rng.next() % 60 for _ in range(11)]
    for mode, det in MODES:
        _cmp(ctx, r1 + r2, w1 + w2, c, mode, det, offsets=offs)  # mixed -> banded
    big = O.cfg(400, 4, 6, 1, 12, 40, 5)  # 100 * 400 > i16 -> scalar fallback
    r3, w3 = _batch(rng, 4, 100, 140)
    for mode, det in MODES:
        _cmp(ctx, r3, w3, big, mode, det, offsets=[0, 5, 10, 20])


def test_reference_batch_cases(ctx):
    # tests/alignment.rs:124-274 through the GPU drop-in.
    bases = b"ACGTTGCTAATCGTGCATGACCTG"
    c = O.cfg(2, 4, 6, 1, 50, 40, 5)
    for count in (1, 4, 5, 16, 17, 33):
        for mode, det in MODES:
            _cmp(ctx, [bases] * count, [bases] * count, c, mode, det, aborts=[0] * count)
    read = b"GATTACAGCTTGAGTCCACG"
    window = b"C" * 100 + read
    c8 = O.cfg(2, 4, 6, 1, 8, 40, 5)
    for reads in ([read], [read, read[:19]]):
        for mode, det in MODES:
            _cmp(ctx, reads, [window] * len(reads), c8, mode, det,
                 offsets=[100] * len(reads), aborts=[-(2**31) // 4] * len(reads))
    for length, reward, offset in [(7, 4681, 0), (8, 4096, 0), (150, 300, 0)]:
        rd = b"G" * length
        ref = b"C" * offset + rd
        cb = O.cfg(reward, 4, 6, 1, 8, 40, 5)
        for mode, det in MODES:
            _cmp(ctx, [rd], [ref], cb, mode, det, offsets=[offset])
