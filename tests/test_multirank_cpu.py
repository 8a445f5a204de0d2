"""Multi-rank host logic on CPU (gloo, world size 2): cost-balanced contiguous
shards cover every pair once, and rank 0's gather of the per-rank results (here
computed by the oracle, standing in for each rank's GPU) equals the unsharded run
bit for bit, CIGAR offsets rebased. A rank that fails is seen by the other as a
collective error within the process-group timeout."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import pyoracle as O


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _workload():
    from kira_ls_aligner_b200 import synth
    return synth.uneven(n_pairs=900, seed=0xD15, ref_len=300_000, q_hi=160, bands=(8, 16, 32))


def _oracle_results(w, lo, hi):
    """kira_sw_result rows + compacted CIGAR ops for pairs [lo, hi), from the oracle."""
    from kira_ls_aligner_b200 import _abi
    res = np.zeros(hi - lo, _abi.SW_RESULT_DTYPE)
    ops = []
    for k, p in enumerate(range(lo, hi)):
        r = w.reads[int(w.read_off[p]):int(w.read_off[p]) + int(w.read_len[p])].tobytes()
        win = w.wins[int(w.win_off[p]):int(w.win_off[p]) + int(w.win_len[p])].tobytes()
        o = O.banded_sw(r, win, int(w.band_offset[p]), O.cfg(1, 4, 6, 1, int(w.bandwidth[p]), 100, 5))
        res[k]["score"], res[k]["ref_start"], res[k]["ref_end"] = o.score, o.ref_start, o.ref_end
        res[k]["read_start"], res[k]["read_end"] = o.read_start, o.read_end
        res[k]["cigar_off"], res[k]["n_cigar"] = len(ops), len(o.cigar)
        res[k]["status"], res[k]["early_abort"] = 3, int(o.early_abort)
        ops += [(n << 4) | "MIDNS".index(c) for n, c in o.cigar]
    return res, np.asarray(ops, np.uint32)


def _rank_main(rank, world, port, q, fail_rank):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        from kira_ls_aligner_b200 import shard
        w = _workload()
        bounds = shard.shard_bounds(shard.pair_cost(w.read_len, w.win_len, w.bandwidth), world)
        lo, hi = bounds[rank]
        if rank == fail_rank:
            raise RuntimeError("rank failed before the gather")
        res, ops = _oracle_results(w, lo, hi)
        g = shard.gather_results(res, ops, dist)
        if rank == 0:
            full_res, full_ops = _oracle_results(w, 0, w.n_pairs)
            q.put(("ok", bounds, bool(np.array_equal(g[0], full_res)),
                   bool(np.array_equal(g[1], full_ops))))
    except Exception as e:  # reported to the parent; the process exits cleanly
        q.put(("error", rank, type(e).__name__, str(e)[:200]))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q, fail_rank))
          for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
    out = []
    while not q.empty():
        out.append(q.get())
    return out


def test_shards_cover_and_balance():
    from kira_ls_aligner_b200 import shard
    rng = np.random.default_rng(4)
    cost = shard.pair_cost(rng.integers(50, 300, 10_000), rng.integers(200, 700, 10_000),
                           rng.choice([16, 32, 64, 128], 10_000))
    for world in (1, 2, 3, 8):
        b = shard.shard_bounds(cost, world)
        assert b[0][0] == 0 and b[-1][1] == len(cost)
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        tot = [cost[lo:hi].sum() for lo, hi in b]
        assert max(tot) - min(tot) <= 2 * cost.max()  # within one pair of even
    assert shard.shard_bounds(cost[:1], 4)[0] == (0, 1)
    assert shard.shard_bounds([], 3) == [(0, 0)] * 3


def test_two_ranks_gather_equals_unsharded():
    out = _run(2)
    ok = [o for o in out if o[0] == "ok"]
    assert ok and not [o for o in out if o[0] == "error"], out
    _, bounds, same_res, same_ops = ok[0]
    assert bounds[0][1] == bounds[1][0] and bounds[0][1] > 0
    assert same_res and same_ops


def test_failed_rank_is_seen_by_the_other():
    out = _run(2, fail_rank=1)
    errs = {o[1]: o for o in out if o[0] == "error"}
    assert 1 in errs and errs[1][2] == "RuntimeError"
    assert 0 in errs  # rank 0's gather ended with an error instead of hanging


def test_bench_two_ranks_dry_run():
    """bench.py --gpus 2 launches two ranks itself (torchrun, 127.0.0.1), shards one
    job between them and gathers every rank's rows on rank 0, through the same code
    the GPU run takes; --dry-run replaces the GPU step (gloo, CPU only)."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2",
                        "--backend", "gloo", "--dry-run", "--reads", "2000", "--ref-len",
                        "200000", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    d = json.loads(line)
    assert d["n_gpus"] == 2 and d["dry_run"]
    assert d["shard"]["rank0_pairs"] == [0, 16000]
    assert d["shard"]["gathered"] == {"pairs": 32000, "cigar_ops": 32000,
                                      "offsets_rebased": True}
