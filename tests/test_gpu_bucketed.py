"""Bucketed banded SW (band classes, per-class shapes, dynamic fetch) and the
one-launch path give identical results, equal to the oracle, on a mixed-length,
mixed-band batch (the uneven configuration's distribution, scaled down)."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu


def test_bucketed_equals_plain_equals_oracle():
    from kira_ls_aligner_b200 import (AlignmentConfig, GpuContext, PairBatch, _abi,
                                      decode_cigar, synth)
    w = synth.uneven(n_pairs=6000, seed=0x5151, ref_len=2_000_000)
    b = PairBatch(w.reads, w.read_off, w.read_len, w.wins, w.win_off, w.win_len,
                  w.band_offset, None, w.bandwidth)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    with GpuContext(0) as ctx:
        L = _abi.lib()
        ctx.check(L.kira_gpu_set_plain(ctx.handle, 0))
        rb, ob, cb = ctx.bsw_batch(b, cfg)
        ctx.check(L.kira_gpu_set_plain(ctx.handle, 1))
        rp, op, cp = ctx.bsw_batch(b, cfg)
    assert cb == cp
    fields = ["score", "ref_start", "ref_end", "read_start", "read_end", "n_cigar", "early_abort"]
    for f in fields:
        assert np.array_equal(rb[f], rp[f]), f
    for p in range(w.n_pairs):
        a, c = int(rb["cigar_off"][p]), int(rp["cigar_off"][p])
        n = int(rb["n_cigar"][p])
        assert np.array_equal(ob[a:a + n], op[c:c + n]), p
    sel = np.arange(0, w.n_pairs, 7)
    # every 7th pair against the oracle, each with its own band
    for k, p in enumerate(sel):
        c = O.cfg(1, 4, 6, 1, int(w.bandwidth[p]), 100, 5)
        r = w.reads[int(w.read_off[p]):int(w.read_off[p]) + int(w.read_len[p])].tobytes()
        win = w.wins[int(w.win_off[p]):int(w.win_off[p]) + int(w.win_len[p])].tobytes()
        o = O.banded_sw(r, win, int(w.band_offset[p]), c)
        got = (int(rb["ref_start"][p]), int(rb["ref_end"][p]), int(rb["read_start"][p]),
               int(rb["read_end"][p]), int(rb["score"][p]))
        assert got == (o.ref_start, o.ref_end, o.read_start, o.read_end, o.score), p
        a = int(rb["cigar_off"][p])
        assert decode_cigar(ob[a:a + int(rb["n_cigar"][p])]) == o.cigar, p
