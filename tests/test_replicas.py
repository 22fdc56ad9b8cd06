"""Multi-GPU bookkeeping of bench.py (the droplet step runs as N independent
replicas): two gloo ranks on the CPU agree on the job time (the slowest
rank's), compute the job throughput from every rank's units, and only rank 0
runs the CPU reference arm.  Rendezvous on 127.0.0.1."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from asd2_b200 import replicas as R
    dist = R.init_group("gloo", timeout_s=60)
    local = [1.5, 2.25][rank]
    t = R.job_time(local, dist)
    rate = R.job_rate(10, world, t)
    dist.barrier()
    out.put((rank, t, rate, R.reference_rank_runs(R.rank_env()[0])))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.25, 2.25]           # the slowest rank's time
    assert all(abs(r[2] - 2 * 10 / 2.25) < 1e-12 for r in res)
    assert [r[3] for r in res] == [True, False]          # reference arm on rank 0 only


def test_single_rank_is_plain():
    from asd2_b200 import replicas as R
    assert R.job_time(3.0, None) == 3.0
    assert R.job_rate(5, 1, 2.0) == 2.5
