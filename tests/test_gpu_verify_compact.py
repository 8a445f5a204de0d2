"""Compact result form of the composed verification (kira_gpu_verify_batch_compact):
one status byte per pair plus the rows of the pairs with an alignment, in pair
order -- identical to the full rows of kira_gpu_verify_batch, on the one-shot and
the chunked host path, with the row-capacity error reporting the need."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _compact(ctx, b, params, rows_cap, cigar_cap):
    from kira_ls_aligner_b200 import _abi
    n = b.n
    status = np.zeros(n, np.uint8)
    rows = np.zeros(max(rows_cap, 1), _abi.SW_RESULT_DTYPE)
    ops = np.zeros(cigar_cap, np.uint32)
    cb = _abi.CigarBuf(_abi.ptr(ops), cigar_cap, 0)
    used, cells = C.c_uint64(), C.c_uint64()
    pc, vp = b.to_c(), params.to_c()
    rc = _abi.lib().kira_gpu_verify_batch_compact(ctx.handle, C.byref(pc), C.byref(vp),
                                                  _abi.ptr(status), _abi.ptr(rows), rows_cap,
                                                  C.byref(used), C.byref(cb), C.byref(cells))
    return rc, status, rows[:min(used.value, rows_cap)], used.value, ops[:cb.used], int(
        cells.value)


@pytest.mark.parametrize("n_reads", [5_000, 100_000])  # one-shot, chunked (800k pairs)
def test_compact_equals_full_rows(ctx, n_reads):
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, synth
    w = synth.batched(n_reads=n_reads, ref_len=20_000_000)
    ctx.ref_upload(w.reference)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    res, ops, _, cells = ctx.verify_batch(b, params)
    keep = np.nonzero((res["status"] == 1) | (res["status"] == 3))[0]
    rc, status, rows, used, ops2, cells2 = _compact(ctx, b, params, b.n, len(ops) + 16)
    assert rc == 0
    assert np.array_equal(status, res["status"])
    assert used == len(keep)
    assert np.array_equal(rows.view(np.uint8), res[keep].view(np.uint8))
    assert np.array_equal(ops2, ops) and cells2 == cells
    # too few rows: the status bytes and the need come back, with the capacity error
    rc, status3, rows3, used3, _, _ = _compact(ctx, b, params, len(keep) // 2, len(ops) + 16)
    assert rc == 9 and used3 == len(keep)
    assert np.array_equal(status3, res["status"])
    assert np.array_equal(rows3.view(np.uint8), res[keep[:len(keep) // 2]].view(np.uint8))
