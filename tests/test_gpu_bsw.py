"""GPU banded SW (banded_sw_public per pair) vs the oracle's banded_sw_with:
score, end coordinates, CIGAR, early-abort flag and executed cells, bit-exact."""
import pytest

import pyoracle as O
from gpu_cases import oracle_sw, sw_corpus
from refgen import gen_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _gpu(ctx, cases, cfg):
    from kira_ls_aligner_b200 import PairBatch, results_to_list
    b = PairBatch.from_pairs([c[0] for c in cases], [c[1] for c in cases],
                             band_offset=[c[2] for c in cases],
                             abort_score=[c[4] for c in cases],
                             bandwidth=[c[3] for c in cases])
    res, ops, cells = ctx.bsw_batch(b, cfg)
    return results_to_list(res, ops), cells


def _compare(ctx, cases, cfg):
    got, cells = _gpu(ctx, cases, cfg)
    want = oracle_sw(cases, cfg, adaptive=cfg.adaptive, max_drift=cfg.max_drift,
                     dp_xdrop=(cfg.dp_xdrop if cfg.dp_xdrop >= 0 else cfg.xdrop))
    for i, (g, w) in enumerate(zip(got, want)):
        assert g.key() == w.key(), (i, cases[i][2:], g, w)
    assert cells == sum(w.cells for w in want)


def test_reference_known_answers(ctx):
    from kira_ls_aligner_b200 import AlignmentConfig
    ref = gen_ref(120)
    cases = [
        (ref[0:30] + ref[33:60] + ref[63:120], ref, 0, 4, O.ABORT_DISABLED),  # mod.rs:2368
        (ref[10:90], ref, 10, 6, O.ABORT_DISABLED),                            # mod.rs:2421
        (gen_ref(80)[0:60], gen_ref(80), 0, 8, O.ABORT_DISABLED),              # mod.rs:2483
    ]
    r90 = gen_ref(90)
    cases.append((r90[:40] + b"TTGCA" + r90[40:], r90, 0, 20, O.ABORT_DISABLED))  # mod.rs:2591
    for adaptive in (True, False):
        _compare(ctx, cases, AlignmentConfig(1, 4, 6, 1, 4, 1000, 5, adaptive))
    got, _ = _gpu(ctx, cases[2:3], AlignmentConfig(1, 4, 6, 1, 8, 1000, 5, True))
    assert (got[0].read_start, got[0].read_end, got[0].score) == (0, 60, 60)


@pytest.mark.parametrize("seed,adaptive,xdrop,clip", [
    (0x5CA1AB1E, True, 100, 5), (0xBADA55, False, 100, 5), (0xC0DE, True, 12, 5),
    (0xF00D, True, 100, 0), (0x7777, False, 7, 0)])
def test_random_corpus(ctx, seed, adaptive, xdrop, clip):
    from kira_ls_aligner_b200 import AlignmentConfig
    cases = sw_corpus(seed, 1500)
    _compare(ctx, cases, AlignmentConfig(1, 4, 6, 1, 33, xdrop, clip, adaptive))


def test_wide_bands_and_scoring(ctx):
    from kira_ls_aligner_b200 import AlignmentConfig
    cases = sw_corpus(0xA1B2, 400, qmin=50, qmax=400, pad=300, max_band=271)
    _compare(ctx, cases, AlignmentConfig(2, 3, 5, 2, 33, 60, 5, True, 16))
    cases = sw_corpus(0xA1B3, 400, qmin=1, qmax=60, pad=20, max_band=8)
    _compare(ctx, cases, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 3))


def test_non_acgt_bytes(ctx):
    # SW compares raw bytes: N matches N, lower case differs from upper case.
    from kira_ls_aligner_b200 import AlignmentConfig
    cases = sw_corpus(0xACE, 500, alpha=b"ACGTNacgtRY")
    _compare(ctx, cases, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True))


def test_empty_and_degenerate(ctx):
    from kira_ls_aligner_b200 import AlignmentConfig
    cases = [(b"A", b"A", 0, 1, O.ABORT_DISABLED), (b"ACGT", b"TTTT", 0, 2, O.ABORT_DISABLED),
             (b"ACGTACGT", b"AC", 0, 3, O.ABORT_DISABLED),
             (b"ACGTACGTAA", b"GGGGGGGGGGGGGACGTACGTAA", 50, 3, O.ABORT_DISABLED),
             (b"ACGTACGTAA", b"ACGTACGTAAGGG", -30, 3, O.ABORT_DISABLED),
             (b"", b"ACGT", 0, 2, O.ABORT_DISABLED)]
    _compare(ctx, cases, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True))
