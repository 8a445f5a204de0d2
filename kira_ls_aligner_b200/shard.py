"""Multi-GPU sharding of a pair batch: one process per GPU, no data-path collective.

Pairs are independent, so each rank verifies a contiguous range of the batch
against its own replica of the resident reference. Ranges are balanced by an
estimate of each pair's DP work (read length x band cells, or x window length
for the full-window mode), and the per-rank results come back to rank 0 with
one gather at the end (sizes first, then the padded payloads), rebasing each
rank's CIGAR offsets onto the concatenated op array.
"""
from __future__ import annotations

import numpy as np

from . import _abi as A
from .runtime import PairBatch


def pair_cost(read_len, win_len, bandwidth=None, band: int = 33) -> np.ndarray:
    """Per-pair work estimate: read bases x cells per row (2 band + 1, capped by the
    window), plus a constant for the per-pair sieve / Myers share."""
    q = np.asarray(read_len, np.float64)
    w = np.asarray(win_len, np.float64)
    b = np.asarray(bandwidth, np.float64) if bandwidth is not None else np.full_like(q, band)
    return q * np.minimum(w, 2.0 * np.maximum(b, 1.0) + 1.0) + 64.0


def shard_bounds(cost, world: int) -> list:
    """Contiguous [lo, hi) ranges, one per rank, with near-equal total cost (every
    pair in exactly one range; ranges may be empty when pairs < ranks)."""
    cost = np.asarray(cost, np.float64)
    n = len(cost)
    if world < 1:
        raise ValueError("world must be >= 1")
    if n == 0:
        return [(0, 0)] * world
    csum = np.cumsum(cost)
    targets = csum[-1] * np.arange(1, world) / world
    cuts = np.searchsorted(csum, targets, side="left") + 1
    cuts = np.clip(cuts, 0, n)
    edges = np.concatenate([[0], np.maximum.accumulate(cuts), [n]]).astype(np.int64)
    return [(int(edges[r]), int(edges[r + 1])) for r in range(world)]


def local_batch(batch: PairBatch, lo: int, hi: int) -> PairBatch:
    """The pairs [lo, hi) of a batch (arenas shared, per-pair arrays sliced)."""
    def sl(a):
        return None if a is None else np.ascontiguousarray(a[lo:hi])
    return PairBatch(batch.read_seq, sl(batch.read_off), sl(batch.read_len), batch.win_seq,
                     sl(batch.win_off), sl(batch.win_len), sl(batch.band_offset),
                     sl(batch.abort_score), sl(batch.bandwidth))


def gather_results(res: np.ndarray, ops: np.ndarray, dist, device=None):
    """Concatenate every rank's (results, CIGAR ops) on rank 0, in rank order, with
    cigar_off rebased onto the gathered op array. Returns (res, ops) on rank 0 and
    (None, None) elsewhere. `dist` is torch.distributed; `device` the tensor device
    the backend needs (None = CPU, as gloo uses)."""
    import torch

    rank, world = dist.get_rank(), dist.get_world_size()
    rb = np.ascontiguousarray(res).view(np.uint8).reshape(-1)
    ob = np.ascontiguousarray(ops).view(np.uint8).reshape(-1)
    sizes = torch.tensor([rb.size, ob.size], dtype=torch.int64, device=device)
    all_sizes = [torch.zeros(2, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(all_sizes, sizes)
    all_sizes = [tuple(int(v) for v in s.cpu()) for s in all_sizes]
    cap = max(a + b for a, b in all_sizes)
    buf = torch.zeros(cap, dtype=torch.uint8, device=device)
    buf[: rb.size] = torch.from_numpy(rb.copy()).to(buf.device)
    buf[rb.size: rb.size + ob.size] = torch.from_numpy(ob.copy()).to(buf.device)
    outs = [torch.zeros(cap, dtype=torch.uint8, device=device) for _ in range(world)] \
        if rank == 0 else None
    dist.gather(buf, outs, dst=0)
    if rank != 0:
        return None, None
    res_parts, op_parts, base = [], [], 0
    for (nr, no), t in zip(all_sizes, outs):
        raw = t.cpu().numpy()
        r = raw[:nr].copy().view(A.SW_RESULT_DTYPE)
        o = raw[nr:nr + no].copy().view(np.uint32)
        r["cigar_off"] += np.uint32(base)
        base += len(o)
        res_parts.append(r)
        op_parts.append(o)
    return np.concatenate(res_parts), np.concatenate(op_parts)
