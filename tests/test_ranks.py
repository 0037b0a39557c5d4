"""The multi-rank path on the CPU: two gloo ranks.

Ranks never exchange data on this path; what runs across ranks is the
barrier, the max over ranks of the timed region, the sum of units, and the
per-rank seeding that gives each rank its own batch.  Two processes with the
gloo backend check each of these, then check that each rank's own batch is
processed correctly: every rank runs the oracle restatement of the spliced DP
on its shard and the whole-job checksum, gathered over ranks, equals the
single-process result over the union of the shards.  A second test splits ONE
batch with the group planner (pl_group_plan), each rank aligns its share, rank 0
gathers the shares (the only exchange, on the host) and reassembles them with
pl_group_gather: the result equals a single process's over the whole batch.
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


def _batch_pairs():
    from protlocus_b200 import workload as W
    rng = np.random.default_rng(77)
    return [W.random_pair(rng, max_al=40) for _ in range(14)]


def _align(pairs):
    import oracle_lib as O
    from protlocus_b200.abi import NS_F_CIGAR, Options
    opt = Options(flag=NS_F_CIGAR)
    out = []
    for nt, aa in pairs:
        score, _ntl, _aal, cig = O.run("gs_auto", nt, aa, opt)
        out.append((score, [int(x) for x in cig]))
    return out


def _job_table(pairs):
    from protlocus_b200.abi import SpliceJob
    jobs = (SpliceJob * len(pairs))()
    pn = pa = 0
    for q, (nt, aa) in enumerate(pairs):
        jobs[q].nt_off, jobs[q].aa_off, jobs[q].ss_off, jobs[q].nl, jobs[q].al = pn, pa, -1, len(nt), len(aa)
        pn += len(nt)
        pa += len(aa)
    return jobs


def _shard_worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from protlocus_b200 import lib as L
    from protlocus_b200.ranks import Ranks
    R = Ranks("gloo", timeout_s=60)
    try:
        pairs = _batch_pairs()                       # every rank holds the same job table
        dev, _cells = L.group_plan(_job_table(pairs), world)
        mine = _align([pairs[q] for q in range(len(pairs)) if dev[q] == rank])
        shares = [None] * world
        dist.all_gather_object(shares, mine)         # the host-side gather of results
        if rank == 0:
            res, cig, total = L.group_gather(dev, shares)
            out[0] = ([(res[q].score, cig[res[q].cigar_off:res[q].cigar_off + res[q].n_cigar].tolist())
                       for q in range(len(pairs))], dev.tolist())
        R.barrier()
    finally:
        R.close()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_shard_one_batch():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_shard_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        got, dev = out[0]
    assert set(dev) == {0, 1}                        # both ranks took a share
    assert got == _align(_batch_pairs())             # job order and CIGARs as one process
