"""Serving mode (kira_server): continuous batching over several slots. Each
request's results through the server, mixed with other requests, equal the
direct call on that request alone; bounded waits time out with a status; a
failing batch reports its error and the server keeps serving."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _verify_requests(w, sizes):
    from kira_ls_aligner_b200 import PairBatch
    out, at = [], 0
    for n in sizes:
        sl = slice(at, at + n)
        out.append(PairBatch(w.reads, w.read_off[sl].copy(), w.read_len[sl].copy(), None,
                             w.win_off[sl].copy(), w.win_len[sl].copy()))
        at += n
    return out


def _bsw_requests(u, sizes):
    from kira_ls_aligner_b200 import PairBatch
    out, at = [], 0
    for n in sizes:
        sl = slice(at, at + n)
        out.append(PairBatch(u.reads, u.read_off[sl].copy(), u.read_len[sl].copy(), u.wins,
                             u.win_off[sl].copy(), u.win_len[sl].copy(),
                             u.band_offset[sl].copy(), None, u.bandwidth[sl].copy()))
        at += n
    return out


def _same(a, b):
    ra, oa = a
    rb, ob = b
    assert np.array_equal(ra, rb)
    assert np.array_equal(oa, ob)


def test_mixed_requests_equal_alone():
    from kira_ls_aligner_b200 import (AlignmentConfig, GpuContext, Server, VerifyParams,
                                      synth)
    w = synth.make_workload("s", 6000, 400_000, cands=4, sub_lo=0.0, sub_hi=0.04, seed=31)
    u = synth.uneven(n_pairs=4000, seed=0x77, ref_len=1_000_000)
    vreq = _verify_requests(w, [700, 1500, 300, 2500, 1200, 4000, 900, 2000, 600, 3000])
    breq = _bsw_requests(u, [400, 900, 150, 1200, 600, 750])
    vp = VerifyParams(sieve_threshold=12, myers_k=8)
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    alone_v, alone_b = [], []
    with GpuContext(0) as ctx:
        ctx.ref_upload(w.reference)
        for b in vreq:
            r, o, _, _ = ctx.verify_batch(b, vp)
            alone_v.append((r, o))
        for b in breq:
            r, o, _ = ctx.bsw_batch(b, cfg)
            alone_b.append((r, o))
    with Server(0, slots=3, max_batch_pairs=6000) as srv:
        srv.ref_upload(w.reference)
        tickets = []
        lock = threading.Lock()

        def feed(reqs, kind):
            for i, b in enumerate(reqs):
                t = srv.submit_verify(b, vp) if kind == "v" else srv.submit_bsw(b, cfg)
                with lock:
                    tickets.append((kind, i, t))

        th = [threading.Thread(target=feed, args=(vreq, "v")),
              threading.Thread(target=feed, args=(breq, "b"))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        infos = []
        for kind, i, t in tickets:
            got = t.wait(120.0)
            _same(got, alone_v[i] if kind == "v" else alone_b[i])
            infos.append(t.info())
        assert srv.stats()["pairs"] == sum(b.n for b in vreq + breq)
    assert all(x.status == 0 and x.t_done_ns >= x.t_start_ns >= x.t_submit_ns for x in infos)
    assert max(x.batch_requests for x in infos) > 1  # requests were batched together


def test_poll_and_bounded_wait():
    # One slot: the second request queues behind the first, so it is pending at
    # once and a zero-length wait on it must time out with a status.
    from kira_ls_aligner_b200 import Server, Timeout, VerifyParams, _abi, synth
    w = synth.make_workload("t", 60_000, 2_000_000, cands=8, seed=5)
    half = w.n_pairs // 2
    a, b = _verify_requests(w, [half, w.n_pairs - half])
    vp = VerifyParams(sieve_threshold=12, myers_k=8)
    with Server(0, slots=1, max_batch_pairs=half) as srv:
        srv.ref_upload(w.reference)
        t1 = srv.submit_verify(a, vp)
        t2 = srv.submit_verify(b, vp)
        assert t2.poll() == _abi.KIRA_PENDING
        with pytest.raises(Timeout):
            t2.wait(0.0)
        for t, n in ((t1, half), (t2, w.n_pairs - half)):
            res, ops = t.wait(120.0)
            assert len(res) == n and t.done()
            t.release()


def test_capacity_and_errors_do_not_stop_the_server():
    from kira_ls_aligner_b200 import (AlignmentConfig, CapacityError, InvalidArgument, Server,
                                      synth)
    u = synth.uneven(n_pairs=600, seed=0x99, ref_len=500_000)
    good, other = _bsw_requests(u, [300, 300])
    with Server(0, slots=2) as srv:
        t = srv.submit_bsw(good, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16),
                           cigar_cap=4)
        with pytest.raises(CapacityError):
            t.wait(60.0)
        assert t.info().cigar_used > 4
        bad = srv.submit_bsw(other, AlignmentConfig(1, 4, -6, 1, 33, 100, 5, True, 16))
        with pytest.raises(InvalidArgument):
            bad.wait(60.0)
        ok = srv.submit_bsw(other, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16))
        res, ops = ok.wait(60.0)
        assert (res["status"] == 3).all() and len(ops) > 0
