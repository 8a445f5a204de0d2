"""kira_gpu_bsw_batch_noalloc, the allocation-free banded SW entry point, called
through the C ABI: its results must equal kira_gpu_bsw_batch's, bit for bit, on
two calls in a row (the second with a different batch shape, so anything the
first call left in the shared scratch array must not leak into it).

This entry point exists for callers that cannot allocate device memory (their
memory belongs to another allocator, or cudaMalloc's device-wide synchronisation
is not acceptable on their path); it keeps all scratch in one fixed device array
of the library. The file name makes pytest collect it last."""
import ctypes as C

import numpy as np
import pytest

import pyoracle as O
from gpu_cases import sw_corpus

pytestmark = pytest.mark.gpu


def _dev_batch(cases, torch, dev):
    from kira_ls_aligner_b200 import PairBatch, _abi
    b = PairBatch.from_pairs([c[0] for c in cases], [c[1] for c in cases],
                             band_offset=[c[2] for c in cases],
                             abort_score=[c[4] for c in cases],
                             bandwidth=[c[3] for c in cases])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    keep = {
        "read_seq": t(np.concatenate([b.read_seq, np.zeros(16, np.uint8)])),
        "win_seq": t(np.concatenate([b.win_seq, np.zeros(16, np.uint8)])),
        "read_off": t(b.read_off.view(np.int64)), "read_len": t(b.read_len.view(np.int32)),
        "win_off": t(b.win_off.view(np.int64)), "win_len": t(b.win_len.view(np.int32)),
        "band_offset": t(b.band_offset), "abort_score": t(b.abort_score),
        "bandwidth": t(b.bandwidth),
    }
    p = _abi.Pairs()
    p.n = b.n
    p.max_read_len = int(b.read_len.max())
    p.max_win_len = int(b.win_len.max())
    p.max_bandwidth = int(b.bandwidth.max())
    p.read_seq, p.read_seq_bytes = keep["read_seq"].data_ptr(), int(b.read_seq.nbytes)
    p.win_seq, p.win_seq_bytes = keep["win_seq"].data_ptr(), int(b.win_seq.nbytes)
    for name in ("read_off", "read_len", "win_off", "win_len", "band_offset", "abort_score",
                 "bandwidth"):
        setattr(p, name, keep[name].data_ptr())
    return b, p, keep


SENTINEL = 0x5A5A5A5A


def _noalloc(p, cfg, n, cap, torch, dev, ops_len=None, full=False):
    """One call; returns (results, ops[:used]) or, with full=True, (results, every op
    word of the buffer, used)."""
    from kira_ls_aligner_b200 import _abi
    out = torch.zeros(n * 32, dtype=torch.uint8, device=dev)
    ops = torch.full((ops_len or cap,), SENTINEL, dtype=torch.int32, device=dev)
    used = torch.zeros(1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    cc = cfg.to_c()
    rc = _abi.lib().kira_gpu_bsw_batch_noalloc(C.byref(p), C.byref(cc), out.data_ptr(),
                                                ops.data_ptr(), cap, used.data_ptr(),
                                                C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize(dev)
    assert rc == 0, rc
    u = int(used.item())
    res = np.frombuffer(out.cpu().numpy().tobytes(), _abi.SW_RESULT_DTYPE)
    allops = ops.cpu().numpy().view(np.uint32)
    if full:
        return res, allops, u
    assert u <= cap
    return res, allops[:u]


def test_noalloc_matches_bsw_batch_on_two_calls():
    torch = pytest.importorskip("torch")
    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext, results_to_list
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    batches = [sw_corpus(0x0A11C, 600, qmin=20, qmax=200, pad=60, max_band=48),
               sw_corpus(0x0A11D, 300, qmin=100, qmax=400, pad=200, max_band=120)]
    with GpuContext(0) as ctx:
        for cases in batches:  # two calls in a row, different shapes
            b, p, keep = _dev_batch(cases, torch, dev)
            want_res, want_ops, _ = ctx.bsw_batch(b, cfg)
            got_res, got_ops = _noalloc(p, cfg, b.n, 64 * b.n, torch, dev)
            got = results_to_list(got_res, got_ops)
            want = results_to_list(want_res, want_ops)
            assert [g.key() for g in got] == [w.key() for w in want]
            # and both equal the oracle's banded_sw_with on a sample
            for i in range(0, b.n, 50):
                read, win, off, band, abort = cases[i]
                c = O.OrcCfg(1, 4, 6, 1, band, 100, 5)
                o = O.banded_sw(read, win, off, c, abort_score=abort)
                assert got[i].key() == o.key()


def test_noalloc_rejects_batches_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    from kira_ls_aligner_b200 import AlignmentConfig, _abi
    dev = torch.device("cuda", 0)
    cases = sw_corpus(0x0A11E, 4, qmin=100, qmax=120, pad=40, max_band=30)
    b, p, keep = _dev_batch(cases, torch, dev)
    p.n = 4
    p.max_read_len = 600_000  # 4 x 600k rows x 48 B of trace: far beyond the fixed array
    cc = AlignmentConfig(1, 4, 6, 1, 33, 100, 5).to_c()
    out = torch.zeros(4 * 32, dtype=torch.uint8, device=dev)
    ops = torch.zeros(16, dtype=torch.int32, device=dev)
    used = torch.zeros(1, dtype=torch.int64, device=dev)
    rc = _abi.lib().kira_gpu_bsw_batch_noalloc(C.byref(p), C.byref(cc), out.data_ptr(),
                                                ops.data_ptr(), 16, used.data_ptr(), None)
    assert rc == _abi.KIRA_ERR_SCRATCH_LIMIT


def test_noalloc_short_cigar_buffer_reports_the_need():
    """With cigar_cap below the ops the batch produces, *cigar_used still gives the
    full need and nothing is written past cigar_cap."""
    torch = pytest.importorskip("torch")
    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    cases = sw_corpus(0x0A120, 200, qmin=40, qmax=160, pad=50, max_band=40)
    b, p, keep = _dev_batch(cases, torch, dev)
    with GpuContext(0) as ctx:
        _, want_ops, _ = ctx.bsw_batch(b, cfg)
    need = len(want_ops)
    cap = need // 3
    res, allops, used = _noalloc(p, cfg, b.n, cap, torch, dev, ops_len=need + 64, full=True)
    assert used == need > cap
    assert (allops[cap:] == SENTINEL).all()
    # every pair whose ops lie wholly below the cap has them written in place (a pair
    # that straddles the cap is skipped whole)
    ends = res["cigar_off"].astype(np.int64) + res["n_cigar"].astype(np.int64)
    inside = ends[ends <= cap]
    end = int(inside.max()) if len(inside) else 0
    assert end > 0
    assert (allops[:end] == want_ops[:end]).all()


def test_noalloc_reports_pairs_beyond_the_declared_maxima():
    """A pair longer than max_read_len is not aligned: its row carries
    KIRA_PAIR_OUT_OF_BOUNDS with no CIGAR, and every other pair is unchanged."""
    torch = pytest.importorskip("torch")
    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext, _abi, results_to_list
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    # reads of 30-90 bases (at most 96 after the corpus's insertions), pair 17 150
    cases = sw_corpus(0x0A121, 64, qmin=30, qmax=90, pad=50, max_band=40)
    long_read, long_win = cases[0][0] * 2, cases[0][1] * 2
    cases[17] = (long_read[:150], long_win[:220], 0, 20, O.ABORT_DISABLED)
    assert all(len(c[0]) <= 100 for i, c in enumerate(cases) if i != 17)
    b, p, keep = _dev_batch(cases, torch, dev)
    p.max_read_len = 100  # pair 17 (150 bases) exceeds it
    with GpuContext(0) as ctx:
        want_res, want_ops, _ = ctx.bsw_batch(b, cfg)
    got_res, got_ops = _noalloc(p, cfg, b.n, 64 * b.n, torch, dev)
    assert got_res["status"][17] == _abi.KIRA_PAIR_OUT_OF_BOUNDS
    assert got_res["n_cigar"][17] == 0
    got, want = results_to_list(got_res, got_ops), results_to_list(want_res, want_ops)
    others = [i for i in range(b.n) if i != 17]
    assert all(got_res["status"][i] == _abi.KIRA_PAIR_SW for i in others)
    assert [got[i].key() for i in others] == [want[i].key() for i in others]
