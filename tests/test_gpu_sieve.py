"""GPU sieve (CudaBackend.run_batch drop-in) vs the oracle's restatement of
spectral_scan_kernel / scan_best_with_second (tests/cuda_spectral.rs:74-137)."""
import pytest

import pyoracle as O
from refgen import BASES, XorShift
from test_oracle_sieve import cuda_corpus

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from kira_ls_aligner_b200.cuda import CudaBackend
    b = CudaBackend.new()
    yield b
    b.release_buffers()


def _jobs(corpus):
    from kira_ls_aligner_b200.bitpacked import PackedDna
    from kira_ls_aligner_b200.cuda import CudaJob
    jobs = []
    for read, text, mm in corpus:
        pr, pt = PackedDna.pack(read), PackedDna.pack(text)
        jobs.append(CudaJob(pr.bits, len(read), pt.pre_shifted_window(), len(text), mm))
    return jobs


def _check(corpus, results):
    for (read, text, mm), g in zip(corpus, results):
        rb, _, _ = O.pack(read)
        tb, _, _ = O.pack(text)
        s, m, sec = O.gpu_sieve_semantics(rb, len(read), tb, len(text), mm)
        assert (g.shift, g.mismatches) == (s, m), (len(read), len(text))
        assert g.second_mismatches == (None if sec == 2**31 - 1 else sec)


def test_cuda_spectral_corpus(backend):
    corpus = cuda_corpus(64)
    _check(corpus, backend.run_batch(_jobs(corpus)))


def test_random_lengths_and_tails(backend):
    rng = XorShift(0x51EE)
    corpus = []
    for _ in range(3000):
        r = 1 + rng.next() % 256
        w = r + rng.next() % 300
        read = bytes(BASES[rng.next() % 4] for _ in range(r))
        text = bytearray(BASES[rng.next() % 4] for _ in range(w))
        if rng.next() % 2:
            s = rng.next() % (w - r + 1)
            text[s:s + r] = read
            for _ in range(rng.next() % 5):
                p = s + rng.next() % r
                text[p] = ord("T") if text[p] == ord("A") else ord("A")
        corpus.append((read, bytes(text), rng.next() % 12))
    _check(corpus, backend.run_batch(_jobs(corpus)))


def test_edge_cases(backend):
    corpus = [(b"ACGT", b"ACG", 5), (b"ACGT", b"ACGT", 0), (b"ACGT", b"ACGTACGT", 0),
              (b"A", b"A", 0), (b"AAAAAAAA", b"TTTTTTTTTTTT", 3),
              (b"ACGTACGT", b"AAAAACGTACGTAAAA", 0)]
    _check(corpus, backend.run_batch(_jobs(corpus)))
    assert backend.run_batch([]) == []


def test_read_too_long(backend):
    from kira_ls_aligner_b200.cuda import CudaJob, ReadTooLong
    with pytest.raises(ReadTooLong):
        backend.run_batch([CudaJob(bytes(65), 260, [bytes(80)] * 4, 300, 5)])


def test_dispatcher_roundtrip():
    from kira_ls_aligner_b200.cuda import dispatcher
    corpus = cuda_corpus(16)
    dispatcher.start()
    try:
        res = dispatcher.dispatch(_jobs(corpus))
        assert res is not None
        _check(corpus, res)
    finally:
        dispatcher.stop()
