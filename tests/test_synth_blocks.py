"""The multi-block batched job: block 0 is the one-block workload itself, and any
pair range of the job carries exactly the pairs of the blocks it covers (the
ranges each rank of a multi-GPU run generates for itself)."""
import numpy as np

from kira_ls_aligner_b200 import synth

BP, REF = 16_000, 200_000  # pairs per block, reference bases (small stand-ins)


def _pair_bytes(w, i):
    o, n = int(w.read_off[i]), int(w.read_len[i])
    return bytes(w.reads[o:o + n]), int(w.win_off[i]), int(w.win_len[i])


def test_block_zero_is_the_one_block_workload():
    a = synth.batched(n_reads=BP // 8, ref_len=REF)
    b = synth.batched_range(0, BP, block_pairs=BP, ref_len=REF)
    assert np.array_equal(a.reference, b.reference)
    assert np.array_equal(a.reads, b.reads)
    for f in ("read_off", "read_len", "win_off", "win_len", "is_true"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_ranges_concatenate_the_blocks():
    b0 = synth.batched(n_reads=BP // 8, ref_len=REF)
    b1 = synth.batched(n_reads=BP // 8, ref_len=REF, block=1, ref=b0.reference)
    assert not np.array_equal(b0.reads, b1.reads)
    r = synth.batched_range(10_000, 20_000, block_pairs=BP, ref_len=REF)
    assert r.n_pairs == 10_000
    for k in range(0, 10_000, 97):
        src, i = (b0, 10_000 + k) if 10_000 + k < BP else (b1, 10_000 + k - BP)
        assert _pair_bytes(r, k) == _pair_bytes(src, i)
    # the read arena holds only the reads the range uses
    assert r.reads.nbytes == int(r.read_len.astype(np.int64).sum()) // 8
