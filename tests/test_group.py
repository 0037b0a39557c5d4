"""Sharding one batch over several GPUs, on the CPU: the planner and the gather.

pl_group_plan assigns each job of a caller's table to a device slot (decreasing
DP cells, each to the least-loaded slot); pl_group_gather puts the per-slot
results back in job order with dense CIGARs.  Both are host functions, so the
partition and the reassembly are checked here without a device; the two-rank
gloo test in test_ranks.py runs the same split across processes.
"""
import numpy as np
import pytest

from protlocus_b200 import lib as L
from protlocus_b200.abi import SpliceJob


def _jobs(rng, n):
    jobs = (SpliceJob * n)()
    for q in range(n):
        jobs[q].nl = int(rng.integers(3, 50000))
        jobs[q].al = int(rng.integers(1, 2500))
        jobs[q].ss_off = -1
    return jobs


@pytest.mark.parametrize("n_dev", [1, 2, 3, 8])
def test_plan_assigns_every_job_once_and_balances(n_dev):
    rng = np.random.default_rng(n_dev)
    n = 4000
    jobs = _jobs(rng, n)
    dev, cells = L.group_plan(jobs, n_dev)
    assert dev.shape == (n,) and dev.min() >= 0 and dev.max() < n_dev
    c = np.array([(max(jobs[q].nl - 2, 1)) * jobs[q].al for q in range(n)], np.int64)
    assert np.array_equal(np.bincount(dev, weights=c, minlength=n_dev).astype(np.int64), cells)
    # longest-processing-time order: no slot exceeds another by more than the largest job
    assert cells.max() - cells.min() <= c.max()
    # deterministic
    assert np.array_equal(L.group_plan(jobs, n_dev)[0], dev)


def test_plan_spreads_equal_jobs_round_robin():
    jobs = (SpliceJob * 12)()
    for q in range(12):
        jobs[q].nl, jobs[q].al = 1002, 10
    dev, cells = L.group_plan(jobs, 4)
    assert dev.tolist() == [0, 1, 2, 3] * 3 and (cells == 3 * 1000 * 10).all()


def test_plan_refuses_bad_sizes():
    jobs = (SpliceJob * 1)()
    with pytest.raises(RuntimeError):
        L.group_plan(jobs, 0)
    with pytest.raises(RuntimeError):
        L.group_plan(jobs, 65)


def test_gather_restores_job_order_and_dense_cigars():
    rng = np.random.default_rng(3)
    n, n_dev = 50, 3
    dev = rng.integers(0, n_dev, n).astype(np.int32)
    want = [(int(rng.integers(-100, 1000)), [int(x) for x in rng.integers(0, 1 << 20, int(rng.integers(0, 9)))])
            for _ in range(n)]
    per = [[want[q] for q in range(n) if dev[q] == d] for d in range(n_dev)]
    res, cig, total = L.group_gather(dev, per)
    off = 0
    for q in range(n):
        assert res[q].score == want[q][0] and res[q].status == 0 and res[q].cigar_off == off
        assert cig[off:off + res[q].n_cigar].tolist() == want[q][1]
        off += len(want[q][1])
    assert total == off


def test_gather_marks_jobs_past_the_cigar_buffer():
    dev = np.array([0, 1, 0], np.int32)
    per = [[(5, [1, 2, 3]), (7, [4])], [(6, [9, 9])]]
    res, cig, total = L.group_gather(dev, per, cigar_cap=4)
    assert [res[q].status for q in range(3)] == [0, -2, -2]
    assert cig[:3].tolist() == [1, 2, 3] and total == 6
