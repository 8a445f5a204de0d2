"""CUDA-graph replay of the bucketed banded-SW launches: results with graphs equal
the direct launches, a repeated launch plan replays the cached graph (also with new
sequence content in the same buffers), and a changed plan recaptures."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _counts(ctx):
    from kira_ls_aligner_b200 import _abi
    c, r = C.c_uint64(), C.c_uint64()
    ctx.check(_abi.lib().kira_gpu_set_graphs(ctx.handle, -1, C.byref(c), C.byref(r)))
    return c.value, r.value


def _batch(w, reads=None):
    from kira_ls_aligner_b200 import PairBatch
    return PairBatch(w.reads if reads is None else reads, w.read_off, w.read_len, w.wins,
                     w.win_off, w.win_len, w.band_offset, None, w.bandwidth)


def _same(a, b):
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_graph_replay_equals_direct():
    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext, _abi, synth
    w1 = synth.uneven(n_pairs=5000, seed=0x61, ref_len=1_000_000)
    w2 = synth.uneven(n_pairs=3000, seed=0x62, ref_len=1_000_000)
    # Same lengths, bands and buffers as w1, different bases (complemented reads).
    comp = np.frombuffer(bytes(w1.reads).translate(bytes.maketrans(b"ACGT", b"TGCA")), np.uint8)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    with GpuContext(0) as ctx:
        L = _abi.lib()
        direct = [ctx.bsw_batch(_batch(w1), cfg), ctx.bsw_batch(_batch(w2), cfg),
                  ctx.bsw_batch(_batch(w1, comp), cfg)]
        ctx.check(L.kira_gpu_set_graphs(ctx.handle, 1, None, None))
        c0, r0 = _counts(ctx)
        for _ in range(3):
            _same(ctx.bsw_batch(_batch(w1), cfg), direct[0])
        c1, r1 = _counts(ctx)
        assert c1 - c0 == 1 and r1 - r0 == 2
        _same(ctx.bsw_batch(_batch(w1, comp), cfg), direct[2])  # same plan, new content
        assert _counts(ctx) == (c1, r1 + 1)
        _same(ctx.bsw_batch(_batch(w2), cfg), direct[1])        # new plan: recapture
        assert _counts(ctx)[0] == c1 + 1
        _same(ctx.bsw_batch(_batch(w1), cfg), direct[0])
        ctx.check(L.kira_gpu_set_graphs(ctx.handle, 0, None, None))
        _same(ctx.bsw_batch(_batch(w1), cfg), direct[0])
