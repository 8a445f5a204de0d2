"""NM and MD:Z on the GPU (kira_gpu_nm_md) from the results and CIGARs of the
banded-SW and composed-verification calls, against the oracle's
nm_md_from_cigar (src/alignment/md.rs:162-205) pair by pair: identical NM and
identical MD text, including non-ACGT and lower-case bytes."""
import numpy as np
import pytest

import pyoracle as O
from gpu_cases import sw_corpus

pytestmark = pytest.mark.gpu
NONE = 0xFFFFFFFF


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _oracle(batch, res, ops, win_arena=None):
    out = []
    wins = batch.win_seq if batch.win_seq is not None else win_arena
    for p in range(batch.n):
        r = res[p]
        if r["n_cigar"] == 0:
            out.append((NONE, ""))
            continue
        read = batch.read_seq[int(batch.read_off[p]):int(batch.read_off[p]) + int(batch.read_len[p])]
        win = wins[int(batch.win_off[p]):int(batch.win_off[p]) + int(batch.win_len[p])]
        cig = ops[int(r["cigar_off"]):int(r["cigar_off"]) + int(r["n_cigar"])]
        out.append(O.nm_md(read.tobytes(), win.tobytes(), int(r["read_start"]),
                           int(r["ref_start"]), [int(w) for w in cig]))
    return out


def _check(ctx, batch, res, ops, win_arena=None):
    nm, md = ctx.nm_md(batch, res, ops)
    want = _oracle(batch, res, ops, win_arena)
    for p, (a, b, w) in enumerate(zip(nm, md, want)):
        assert (int(a), b) == w, (p, a, b, w)
    return nm, md


@pytest.mark.parametrize("alpha", [b"ACGT", b"ACGTNacgtRY="])
def test_banded_sw_results(ctx, alpha):
    from kira_ls_aligner_b200 import AlignmentConfig, PairBatch
    cases = sw_corpus(0x3D3D + len(alpha), 800, alpha=alpha)
    b = PairBatch.from_pairs([c[0] for c in cases], [c[1] for c in cases],
                             band_offset=[c[2] for c in cases], abort_score=[c[4] for c in cases],
                             bandwidth=[c[3] for c in cases])
    res, ops, _ = ctx.bsw_batch(b, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16))
    nm, md = _check(ctx, b, res, ops)
    assert any("^" in m for m in md) and any(x > 0 for x in nm)


def test_composed_verification_results(ctx):
    # certified (qM), banded-SW and rejected pairs, resident reference windows
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, synth
    w = synth.make_workload("m", 4000, 300_000, cands=4, sub_lo=0.0, sub_hi=0.05, seed=12)
    ctx.ref_upload(w.reference)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    res, ops, _, _ = ctx.verify_batch(b, VerifyParams(sieve_threshold=12, myers_k=8))
    nm, _ = _check(ctx, b, res, ops, win_arena=w.reference)
    st = res["status"]
    assert {1, 2, 3} <= set(np.unique(st).tolist())
    assert (nm[st == 2] == NONE).all() and (nm[st != 2] != NONE).all()


def test_capacity_and_bad_cigar_range(ctx):
    from kira_ls_aligner_b200 import (AlignmentConfig, CapacityError, InvalidArgument,
                                      PairBatch)
    cases = sw_corpus(0x77, 50)
    b = PairBatch.from_pairs([c[0] for c in cases], [c[1] for c in cases],
                             band_offset=[c[2] for c in cases], bandwidth=[c[3] for c in cases])
    res, ops, _ = ctx.bsw_batch(b, AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16))
    with pytest.raises(CapacityError):
        ctx.nm_md(b, res, ops, md_cap=4)
    bad = res.copy()
    bad["cigar_off"][np.argmax(bad["n_cigar"])] = len(ops) + 5
    with pytest.raises(InvalidArgument):
        ctx.nm_md(b, bad, ops)
