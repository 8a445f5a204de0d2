"""Banded SW in trace rounds: with a trace budget far below the batch's need the
DP sweep and traceback run in many rounds over one reused arena, and every
result equals the single-round run (and the oracle)."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _budget(ctx, nbytes):
    from kira_ls_aligner_b200 import _abi
    ctx.check(_abi.lib().kira_gpu_set_trace_budget(ctx.handle, nbytes))


def _plain(ctx, on):
    from kira_ls_aligner_b200 import _abi
    ctx.check(_abi.lib().kira_gpu_set_plain(ctx.handle, 1 if on else 0))


def _same(a, b):
    ra, oa, ca = a
    rb, ob, cb = b
    assert ca == cb
    for f in ("score", "ref_start", "ref_end", "read_start", "read_end", "n_cigar",
              "early_abort", "status"):
        assert np.array_equal(ra[f], rb[f]), f
    for p in range(len(ra)):
        x, y, n = int(ra["cigar_off"][p]), int(rb["cigar_off"][p]), int(ra["n_cigar"][p])
        assert np.array_equal(oa[x:x + n], ob[y:y + n]), p


@pytest.mark.parametrize("plain", [False, True])
def test_bsw_rounds_equal_single_round(ctx, plain):
    from kira_ls_aligner_b200 import AlignmentConfig, PairBatch, synth
    w = synth.uneven(n_pairs=3000, seed=0x2020, ref_len=1_000_000)
    b = PairBatch(w.reads, w.read_off, w.read_len, w.wins, w.win_off, w.win_len,
                  w.band_offset, None, w.bandwidth)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    _plain(ctx, plain)
    try:
        _budget(ctx, 0)
        one = ctx.bsw_batch(b, cfg)
        _budget(ctx, 3 << 20)  # a few hundred items per round
        many = ctx.bsw_batch(b, cfg)
    finally:
        _budget(ctx, 0)
        _plain(ctx, False)
    _same(one, many)
    res, ops, _ = many
    for p in range(0, w.n_pairs, 29):
        c = O.cfg(1, 4, 6, 1, int(w.bandwidth[p]), 100, 5)
        r = w.reads[int(w.read_off[p]):int(w.read_off[p]) + int(w.read_len[p])].tobytes()
        win = w.wins[int(w.win_off[p]):int(w.win_off[p]) + int(w.win_len[p])].tobytes()
        o = O.banded_sw(r, win, int(w.band_offset[p]), c)
        assert (int(res["score"][p]), int(res["ref_end"][p]), int(res["read_end"][p])) == \
            (o.score, o.ref_end, o.read_end), p


def test_verify_rounds_equal_single_round(ctx):
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, synth
    w = synth.make_workload("r", 4000, 300_000, cands=6, sub_lo=0.0, sub_hi=0.05, seed=7)
    arena, woffs = w.windows_arena()
    b = PairBatch(w.reads, w.read_off, w.read_len, arena, woffs, w.win_len)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    try:
        _budget(ctx, 0)
        r1, o1, _, c1 = ctx.verify_batch(b, params)
        _budget(ctx, 1 << 20)
        r2, o2, _, c2 = ctx.verify_batch(b, params)
    finally:
        _budget(ctx, 0)
    assert (r1["status"] == 3).sum() > 100  # enough SW items to span many rounds
    _same((r1, o1, c1), (r2, o2, c2))
