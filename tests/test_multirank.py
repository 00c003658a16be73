"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

Each rank prices its own shard of calibrations (weak scaling, no data-path
collective); the job's throughput is all ranks' options over the slowest
rank's time; the reference arm runs on rank 0 only."""
import argparse
import importlib
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    bench = importlib.import_module("bench")
    args = argparse.Namespace(workload="uneven", calibs=16, seed=0)
    calibs, _ = bench.workload(args, rank)
    opts = sum(c.outer for c in calibs)
    ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    value, ms_max = bench.job_throughput(ms, opts, 3, world, "cpu")
    total = bench.rank_reduce(opts, "sum", world, "cpu")
    out.put((rank, [(c.numX, c.numY, c.numT, c.outer) for c in calibs], opts, value, ms_max, total))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, shard0, o0, v0, m0, t0), (r1, shard1, o1, v1, m1, t1) = res
    assert shard0 != shard1 and len(shard0) == len(shard1) == 16  # own shard, same size
    assert m0 == m1 == 150.0                                        # max over ranks
    assert t0 == t1 == o0 + o1
    assert v0 == v1 == pytest.approx((o0 + o1) * 3 / 0.150)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    bench = importlib.import_module("bench")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(workload="uneven", calibs=4, seed=0, steps=1, warmup=0, cpu_seconds=0.1, gpus=2)
    bench.run_reference(args)
    assert capsys.readouterr().out == ""
