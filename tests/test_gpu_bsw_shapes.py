"""Every banded-SW launch shape, int32 and packed int16, forced in turn, against
the oracle's banded_sw_with: score, end coordinates, CIGAR, early abort, cells."""
import pytest

from gpu_cases import oracle_sw, sw_corpus

pytestmark = pytest.mark.gpu

CLASS_LOW = (1, 17, 34, 65, 129, 257)  # lowest band of each tuned-shape class


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _force(ctx, shape, cap):
    from kira_ls_aligner_b200 import _abi
    L = _abi.lib()
    for lb in CLASS_LOW:
        ctx.check(L.kira_gpu_set_bsw_shape(ctx.handle, lb, shape if 2 * lb + 1 <= cap else -1))


def _compare(ctx, cases, cfg):
    from kira_ls_aligner_b200 import PairBatch, results_to_list
    b = PairBatch.from_pairs([c[0] for c in cases], [c[1] for c in cases],
                             band_offset=[c[2] for c in cases],
                             abort_score=[c[4] for c in cases],
                             bandwidth=[c[3] for c in cases])
    res, ops, cells = ctx.bsw_batch(b, cfg)
    got = results_to_list(res, ops)
    want = oracle_sw(cases, cfg, adaptive=cfg.adaptive, max_drift=cfg.max_drift,
                     dp_xdrop=(cfg.dp_xdrop if cfg.dp_xdrop >= 0 else cfg.xdrop))
    for i, (g, w) in enumerate(zip(got, want)):
        assert g.key() == w.key(), (i, cases[i][2:], g, w)
    assert cells == sum(w.cells for w in want)


def _shapes():
    from kira_ls_aligner_b200 import autotune
    return list(enumerate(autotune.shapes()))


@pytest.mark.parametrize("shape", range(24))
@pytest.mark.parametrize("scoring", [(1, 4, 6, 1, True, 16), (2, 3, 5, 2, False, 16),
                                     (1, 1, 0, 1, True, 4), (3, 2, 4, 0, True, 16)])
def test_forced_shape(ctx, shape, scoring):
    from kira_ls_aligner_b200 import AlignmentConfig
    shapes = _shapes()
    if shape >= len(shapes):
        pytest.skip("no such shape")
    g, k = shapes[shape][1]
    cap = g * k
    bmax = min((cap - 1) // 2, 280)
    m, x, go, ge, adaptive, drift = scoring
    cases = sw_corpus(0x51A9E + shape * 131 + m, 250, qmin=5, qmax=260, pad=2 * bmax + 20,
                      max_band=bmax)
    _force(ctx, shape, cap)
    try:
        _compare(ctx, cases, AlignmentConfig(m, x, go, ge, 33, 100, 5, adaptive, drift))
    finally:
        _force(ctx, -1, 0)


def test_scores_outside_int16_range_use_int32(ctx):
    # match 12 on 250-base reads leaves the packed range: the batch runs on int32.
    from kira_ls_aligner_b200 import AlignmentConfig
    cases = sw_corpus(0xB16, 200, qmin=150, qmax=250, pad=80, max_band=40)
    _compare(ctx, cases, AlignmentConfig(12, 4, 6, 1, 33, 100, 5, True, 16))
