"""The multi-GPU bench path's host logic, on CPU with two gloo ranks: each
rank simulates its own replica (seed + rank), the job time is the slowest
rank's, the work is summed; the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "dioma-core_b200"))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t, ev = bench.reduce_over_ranks(dist, "cpu", 10.0 + rank, 1000 * (rank + 1))
    args = bench.parse_args_for_test(["--n", "5000", "--k-in", "50"])
    spec, name = bench.workload(args, rank)
    q.put((rank, t, ev, spec["seed"], name))
    dist.destroy_process_group()


def test_two_rank_reduction_and_replica_seeds():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    (r0, t0, e0, s0, n0), (r1, t1, e1, s1, n1) = res
    assert t0 == t1 == 11.0            # the slowest rank's time on every rank
    assert e0 == e1 == 3000.0          # the work of all ranks
    assert s1 == s0 + 1 and n0 == n1   # independent replicas of one workload


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    bench.run_reference(bench.parse_args_for_test(["--impl", "reference"]))
    assert capsys.readouterr().out == ""
