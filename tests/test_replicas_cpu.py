"""Multi-GPU plumbing of the replicas design on CPU: two gloo ranks (the
GPU runs use NCCL with the same calls).  Max-over-ranks timing, sums, the
barrier, and the deterministic partition of an ensemble over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hacc_gpm_b200 import ensemble as E
from hacc_gpm_b200 import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    rk = R.Ranks("gloo", timeout_s=60)
    try:
        rk.barrier()
        mx = rk.allmax(10.0 + rank)        # this rank's "elapsed ms"
        sm = rk.allsum(100.0 * (rank + 1))  # this rank's "particles"
        boxes = E.ensemble_boxes(24)
        parts = R.partition([R.box_cost(b.ng, b.ng, b.nsteps) for b in boxes], world)
        mine = parts[rank]
        n = rk.allsum(len(mine))
        q.put((rank, mx, sm, parts, n))
    finally:
        rk.close()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    (r0, mx0, sm0, parts0, n0), (r1, mx1, sm1, parts1, n1) = res
    assert mx0 == mx1 == 11.0            # the slowest rank's time
    assert sm0 == sm1 == 300.0
    assert parts0 == parts1              # every rank computes the same split
    assert n0 == n1 == 24
    assert sorted(parts0[0] + parts0[1]) == list(range(24))


def _forms_worker(rank, world, port, q):
    from hacc_gpm_b200 import serve as S
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    rk = R.Ranks("gloo", timeout_s=60)
    try:
        boxes = E.shard(E.ensemble_boxes(96), rk.rank, rk.world)
        reqs = E.shard(S.request_stream(160), rk.rank, rk.world)
        got_boxes = rk.gather([(b.tag, b.seed, b.ng, b.rl) for b in boxes])
        got_reqs = rk.gather([(r.tag, r.arrival, r.ng, r.nsteps) for r in reqs])
        q.put((rank, got_boxes, got_reqs))
    finally:
        rk.close()


def test_forms_shard_over_two_gloo_ranks():
    """The ensemble's 96 boxes and the serving stream's 160 requests split
    over two ranks (whole boxes, by predicted cost): every box and request
    lands on exactly one rank, unchanged, and both ranks see the same split
    (what bench.py --workload ensemble|serve runs under torchrun)."""
    from hacc_gpm_b200 import serve as S
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_forms_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    (_, b0, r0), (_, b1, r1) = res
    assert b0 == b1 and r0 == r1
    one_b = sorted((b.tag, b.seed, b.ng, b.rl) for b in E.ensemble_boxes(96))
    one_r = sorted((r.tag, r.arrival, r.ng, r.nsteps) for r in S.request_stream(160))
    assert sorted(b0[0] + b0[1]) == one_b and not set(x[0] for x in b0[0]) & set(x[0] for x in b0[1])
    assert sorted(r0[0] + r0[1]) == one_r and not set(x[0] for x in r0[0]) & set(x[0] for x in r0[1])
    cost = lambda part: sum(R.box_cost(x[2], x[2], 64) for x in part)
    assert max(cost(b0[0]), cost(b0[1])) / min(cost(b0[0]), cost(b0[1])) < 1.1


def test_partition_balances_cost():
    costs = [R.box_cost(b.ng, b.ng, b.nsteps) for b in E.ensemble_boxes(96)]
    parts = R.partition(costs, 4)
    loads = [sum(costs[i] for i in p) for p in parts]
    assert sorted(i for p in parts for i in p) == list(range(96))
    assert max(loads) / min(loads) < 1.05
    assert R.partition(costs, 1) == [list(range(96))]
