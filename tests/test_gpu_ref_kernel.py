"""The reference's own CUDA sieve kernel (src/cuda/spectral.cu, compiled from the
reference source for sm_100a into oracle/_ref/) and the B200 sieve agree on the
same jobs; both are timed on the same batch. Skipped when oracle/_ref was not
built (it needs the reference source tree at build time)."""
import ctypes as C
import os

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


def _flat(jobs):
    n = len(jobs)
    reads = b"".join(j.read_packed for j in jobs)
    refs = b"".join(j.ref_shifted[0] for j in jobs)
    rb = np.array([len(j.read_packed) for j in jobs], np.uint32)
    wb = np.array([len(j.ref_shifted[0]) for j in jobs], np.uint32)
    ro = np.concatenate([[0], np.cumsum(rb)[:-1]]).astype(np.uint64)
    wo = np.concatenate([[0], np.cumsum(wb)[:-1]]).astype(np.uint64)
    return (n, reads, ro, rb, np.full(n, 150, np.uint32), refs, wo, wb,
            np.full(n, 250, np.uint32), np.full(n, 12, np.uint32))


def _reference_run(L, flat):
    """One CudaBackend::run_batch of the reference kernel: (shift, mism, second,
    kernel ms from CUDA events around the launch)."""
    n, reads, ro, rb, rn, refs, wo, wb, wn, mm = flat
    s = np.zeros(n, np.int32)
    m = np.zeros(n, np.int32)
    sec = np.zeros(n, np.int32)
    km, tm = C.c_float(), C.c_float()
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = L.ref_spectral_run_batch(n, reads, p(ro), p(rb), p(rn), refs, p(wo), p(wb), p(wn),
                                  p(mm), p(s), p(m), p(sec), C.byref(km), C.byref(tm))
    assert rc == 0
    return s, m, sec, km.value


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")
def test_reference_kernel_matches():
    from kira_ls_aligner_b200.cuda import CudaBackend
    jobs = _corpus(20000)
    L = C.CDLL(REF_LIB)
    s, m, sec, _ = _reference_run(L, _flat(jobs))
    be = CudaBackend.new()
    ours = be.run_batch(jobs)
    for i, r in enumerate(ours):
        assert (r.shift, r.mismatches) == (s[i], m[i]), i
        assert (r.second_mismatches if r.second_mismatches is not None else 2**31 - 1) == sec[i]


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built")
def test_sieve_kernel_faster_than_reference_kernel():
    """Kernel against kernel on the same device and the same 200k jobs (150-base
    reads, 250-base windows, limit 12): the reference's spectral_scan_kernel (one
    warp per job, the four pre-shifted window copies) and the drop-in sieve kernel
    behind kira_gpu_sieve_batch, each timed with CUDA events around its launch alone
    (median of 5 runs after a warm-up run)."""
    from kira_ls_aligner_b200 import _abi
    from kira_ls_aligner_b200.cuda import CudaBackend
    jobs = _corpus(200_000, seed=0xBEF0)
    flat = _flat(jobs)
    L = C.CDLL(REF_LIB)
    ref_ms = []
    for _ in range(6):
        ref_ms.append(_reference_run(L, flat)[3])
    be = CudaBackend.new()
    ctx = be.context
    lib = _abi.lib()
    ctx.check(lib.kira_gpu_profile(ctx.handle, 1))
    ours_ms = []
    try:
        for _ in range(6):
            be.run_batch(jobs)
            buf = (C.c_float * 4)()
            assert lib.kira_gpu_stage_times(ctx.handle, buf, 4) >= 1
            ours_ms.append(float(buf[0]))
    finally:
        ctx.check(lib.kira_gpu_profile(ctx.handle, 0))
        be.release_buffers()
    ref_k, ours_k = float(np.median(ref_ms[1:])), float(np.median(ours_ms[1:]))
    print(f"\nsieve kernels, 200000 jobs 150x250: reference spectral_scan_kernel "
          f"{ref_k:.4f} ms, B200 sieve_dropin_kernel {ours_k:.4f} ms, ratio {ref_k / ours_k:.2f}")
    assert ours_k < ref_k
