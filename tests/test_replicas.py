"""Runs on several GPUs: the host logic, on CPU ranks of a gloo process group
(world size 2).  The independent systems of the batched workload are split
between the ranks with every system on exactly one rank; the job's time is the
slowest rank's, its work the sum over the ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, weights, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import __graft_entry__ as entry
    rv = entry.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = rv.replicas.shard(weights, rank, world)
    load = sum(weights[i] for i in mine)
    slowest = rv.replicas.max_over_ranks(1.0 + rank, dist)
    total = rv.replicas.sum_over_ranks(load, dist)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, mine, slowest, total))


def test_shard_covers_and_balances(rv):
    w = [float(x) for x in [5, 1, 9, 3, 3, 7, 2, 8, 1, 1]]
    parts = [rv.replicas.shard(w, r, 3) for r in range(3)]
    assert sorted(i for p in parts for i in p) == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert rv.replicas.shard(w, 0, 1) == list(range(len(w)))
    with pytest.raises(ValueError):
        rv.replicas.shard(w, 2, 2)


def test_two_gloo_ranks_split_the_batch(rv):
    fam = rv.problems.batch_family(count=8, seed=2, n_lo=300, n_hi=3000, max_rhs=4)
    weights = [float(rv.SparseLDLT.analyze(s).symbolic.predicted_nnz) for s, _ in fam]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, weights, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, s0, t0), (r1, m1, s1, t1) = res
    assert sorted(m0 + m1) == list(range(len(fam))) and not set(m0) & set(m1)
    assert s0 == s1 == 2.0
    assert t0 == t1 == sum(weights)
