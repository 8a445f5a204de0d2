"""The reference's own CUDA sieve kernel (src/cuda/spectral.cu, compiled from the
reference source for sm_100a into oracle/_ref/) and the B200 sieve agree on the
same jobs; both are timed on the same batch. Skipped when oracle/_ref was not
built (it needs the reference source tree at build time)."""
import ctypes as C
import os
import time

import numpy as np
import pytest

BASES = np.frombuffer(b"ACGT", np.uint8)

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_spectral.so")


def _corpus(n, seed=0xBEEF):
    from kira_ls_aligner_b200.bitpacked import PackedDna
    from kira_ls_aligner_b200.cuda import CudaJob
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        win = BASES[rng.integers(0, 4, 250)].tobytes()
        s = int(rng.integers(0, 101))
        read = bytearray(win[s:s + 150])
        for p in rng.integers(0, 150, int(rng.integers(0, 4))):
            read[p] = ord("T") if read[p] == ord("A") else ord("A")
        pr, pw = PackedDna.pack(bytes(read)), PackedDna.pack(win)
        jobs.append(CudaJob(pr.bits, 150, pw.pre_shifted_window(), 250, 12))
    return jobs


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")
def test_reference_kernel_matches_and_is_slower():
    from kira_ls_aligner_b200.cuda import CudaBackend
    jobs = _corpus(20000)
    n = len(jobs)
    reads = b"".join(j.read_packed for j in jobs)
    refs = b"".join(j.ref_shifted[0] for j in jobs)
    rb = np.array([len(j.read_packed) for j in jobs], np.uint32)
    wb = np.array([len(j.ref_shifted[0]) for j in jobs], np.uint32)
    ro = np.concatenate([[0], np.cumsum(rb)[:-1]]).astype(np.uint64)
    wo = np.concatenate([[0], np.cumsum(wb)[:-1]]).astype(np.uint64)
    rn = np.full(n, 150, np.uint32)
    wn = np.full(n, 250, np.uint32)
    mm = np.full(n, 12, np.uint32)
    s = np.zeros(n, np.int32)
    m = np.zeros(n, np.int32)
    sec = np.zeros(n, np.int32)
    km, tm = C.c_float(), C.c_float()
    L = C.CDLL(REF_LIB)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    for _ in range(2):
        rc = L.ref_spectral_run_batch(n, reads, p(ro), p(rb), p(rn), refs, p(wo), p(wb), p(wn),
                                      p(mm), p(s), p(m), p(sec), C.byref(km), C.byref(tm))
        assert rc == 0
    be = CudaBackend.new()
    be.run_batch(jobs[:64])
    t = time.perf_counter()
    ours = be.run_batch(jobs)
    ours_ms = (time.perf_counter() - t) * 1e3
    for i, r in enumerate(ours):
        assert (r.shift, r.mismatches) == (s[i], m[i]), i
        assert (r.second_mismatches if r.second_mismatches is not None else 2**31 - 1) == sec[i]
    print(f"\nreference spectral_scan_kernel: kernel {km.value:.3f} ms, run_batch "
          f"{tm.value:.3f} ms; B200 run_batch (host API) {ours_ms:.3f} ms for {n} jobs")
