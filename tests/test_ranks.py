"""The multi-rank host logic on the CPU: world size 2 over gloo (as torchrun
would launch it, one process per rank), the rank plumbing bench.py uses
(barrier, maximum over ranks, gather) and the cost partition that shards
the batched workload's independent problems over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ofeli_b200 import problems


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    from ofeli_b200 import ranks
    try:
        R = ranks.Ranks("gloo", torch.device("cpu"), timeout_s=60)
        R.barrier()
        mx = R.max(10.0 + rank)
        costs = problems.batch_costs(1234, 1024)
        mine = problems.partition_by_cost(costs, world)[rank]
        every = R.gather(mine.tolist())
        loads = R.gather(float(costs[mine].sum()))
        R.close()
        q.put((rank, mx, every, loads, None))
    except Exception as e:  # reported to the test
        q.put((rank, None, None, None, repr(e)))


def test_partition_covers_and_balances():
    costs = problems.batch_costs(1234, 1024)
    for parts in (1, 2, 3, 8):
        sh = problems.partition_by_cost(costs, parts)
        allidx = np.concatenate(sh)
        assert np.array_equal(np.sort(allidx), np.arange(1024))
        loads = np.array([costs[s].sum() for s in sh])
        assert loads.max() <= 1.01 * loads.mean()
        assert all(np.all(np.diff(s) > 0) for s in sh)
    assert problems.partition_by_cost([5, 1, 1, 1, 1, 1], 2)[0].tolist() == [0]


@pytest.mark.timeout(300)
def test_two_ranks_over_gloo():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    for rank, mx, every, loads, err in out:
        assert err is None, err
        assert mx == 11.0                              # the maximum over ranks, on every rank
        got = np.sort(np.concatenate([np.array(e) for e in every]))
        assert np.array_equal(got, np.arange(1024))    # each problem solved by exactly one rank
        assert max(loads) <= 1.01 * (sum(loads) / world)
    assert out[0][2] == out[1][2]
