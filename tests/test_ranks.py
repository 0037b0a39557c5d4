"""The multi-rank path on the CPU: two gloo ranks.

Ranks never exchange data on this path; what runs across ranks is the
barrier, the max over ranks of the timed region, the sum of units, and the
per-rank seeding that gives each rank its own batch.  Two processes with the
gloo backend check each of these, then check that each rank's own batch is
processed correctly: every rank runs the oracle restatement of the spliced DP
on its shard and the whole-job checksum, gathered over ranks, equals the
single-process result over the union of the shards.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard(seed):
    from protlocus_b200 import workload as W
    rng = np.random.default_rng(seed)
    return [W.random_pair(rng, max_al=40) for _ in range(6)]


def _checksum(pairs):
    import oracle_lib as O
    from protlocus_b200.abi import NS_F_CIGAR, Options
    opt = Options(flag=NS_F_CIGAR)
    acc = 0
    for nt, aa in pairs:
        score, _ntl, _aal, cig = O.run("gs_auto", nt, aa, opt)
        acc = (acc * 1000003 + (score & 0xFFFFFFFF) + 7 * len(cig)) % (1 << 61)
    return acc


def _worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from protlocus_b200.ranks import Ranks, job_rate
    R = Ranks("gloo", timeout_s=60)
    try:
        assert (R.rank, R.world, R.is_root) == (rank, world, rank == 0)
        R.barrier()
        t = R.max(0.5 + rank)          # slowest rank's time
        u = R.sum(100 * (rank + 1))    # all ranks' units
        seed = R.seed(1)
        pairs = _shard(seed)
        chk = _checksum(pairs)
        gathered = [None] * world
        dist.all_gather_object(gathered, (seed, chk, [len(a) for _, a in pairs]))
        out[rank] = (t, u, job_rate(u, t), gathered)
    finally:
        R.close()


@pytest.mark.timeout(300)
def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank in range(world):
        t, u, rate, gathered = res[rank]
        assert t == 1.5 and u == 300.0 and rate == 200.0
        seeds = [g[0] for g in gathered]
        assert seeds == [1, 2]                      # distinct batches per rank
        assert gathered[0][2] != gathered[1][2]     # and they differ
        # each rank's checksum equals a single process's over the same shard
        for seed, chk, _ in gathered:
            assert chk == _checksum(_shard(seed))
    assert res[0][3] == res[1][3]


def test_single_process_needs_no_process_group(monkeypatch):
    from protlocus_b200.ranks import Ranks, job_rate
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    R = Ranks("gloo")
    assert (R.rank, R.world, R.is_root, R.seed(5)) == (0, 1, True, 5)
    assert R.max(2.5) == 2.5 and R.sum(7) == 7.0
    R.barrier()
    R.close()
    assert job_rate(10, 0) == 0.0
