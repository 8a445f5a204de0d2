"""Long-read gap-fill shape: segments of 200-2000 bases at 5-12 % error, band 256
(513-cell rows, int32 lanes: the scores leave the packed int16 range), windows
taken from a device-resident reference, run in trace rounds (a trace budget far
below the batch's need) -- every pair against the oracle's banded_sw_with,
score, ends, flags and CIGAR op for op."""
import os

import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
NTHREADS = os.cpu_count() or 4


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _check_all(res, ops, cells, out, cig):
    for f in ("score", "ref_start", "ref_end", "read_start", "read_end", "n_cigar",
              "early_abort"):
        bad = np.nonzero(res[f].astype(np.int64) != out[f].astype(np.int64))[0]
        assert len(bad) == 0, (f, bad[:5])
    n = res["n_cigar"].astype(np.int64)
    sel = np.nonzero(n)[0]
    cnt = n[sel]
    pair = np.repeat(sel, cnt)
    t = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    got = ops[res["cigar_off"][pair].astype(np.int64) + t]
    bad = np.nonzero(got != cig[pair, t])[0]
    assert len(bad) == 0, ("cigar", np.unique(pair[bad])[:5])
    assert cells == int(out["cells"].sum())


@pytest.mark.parametrize("budget_mb", [0, 24])
def test_gapfill_band256_every_pair(ctx, budget_mb):
    from kira_ls_aligner_b200 import AlignmentConfig, PairBatch, _abi, synth
    g = synth.gapfill(n_segments=300, seg_lo=200, seg_hi=2000, band=256, ref_len=3_000_000)
    cfg = AlignmentConfig(1, 4, 6, 1, 256, 100, 5, True, 16)
    ctx.ref_upload(g.reference)
    b = PairBatch(g.reads, g.read_off, g.read_len, None, g.win_off, g.win_len, g.band_offset,
                  None, g.bandwidth)
    # 24 MiB of trace slots for ~300 items of up to 2000 rows x 513 int32 cells (4 bits
    # each) forces several rounds over the same arena
    ctx.check(_abi.lib().kira_gpu_set_trace_budget(ctx.handle, budget_mb << 20))
    try:
        res, ops, cells = ctx.bsw_batch(b, cfg)
    finally:
        ctx.check(_abi.lib().kira_gpu_set_trace_budget(ctx.handle, 0))
    need = int(g.read_len.max() + 1) * 257 * 300 // 1  # bytes of one round for every item
    assert budget_mb == 0 or need > 4 * (budget_mb << 20)
    c = O.cfg(1, 4, 6, 1, 256, 100, 5)
    out, cig = O.banded_sw_batch(g.reads, g.read_off, g.read_len, g.reference, g.win_off,
                                 g.win_len, g.band_offset, c, NTHREADS, 2048)
    assert int(out["n_cigar"].max()) <= 2048
    _check_all(res, ops, cells, out, cig)
    assert (res["score"] > 0).mean() > 0.9
