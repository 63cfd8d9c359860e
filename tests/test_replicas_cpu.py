"""Multi-rank host logic of the benchmark on CPU (gloo, world size 2): each
rank runs its own replica (the path has no exchange step), the job's time is
the slowest rank's, and the value counts every rank's sites. Also the
reference arm's rank gating (only rank 0 prints)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(REPO))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    local_ms = [12.5, 20.0][rank]
    m = bench.max_over_ranks(local_ms, dist, "cpu")
    rate = bench.whole_job_rate(21233664, 600, world, m)
    q.put((rank, m, rate))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate in out:
        assert m == 20.0
        assert rate == pytest.approx(2 * 21233664 * 600 / 0.020)


def test_single_rank_identity():
    sys.path.insert(0, str(REPO))
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.whole_job_rate(10, 4, 1, 1000.0) == 40.0


def test_reference_arm_other_ranks_exit_quietly(capsys, monkeypatch):
    sys.path.insert(0, str(REPO))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps = 1
        warmup = 3
        gpus = 2
    assert bench.run_reference_arm(A()) == 0
    assert capsys.readouterr().out == ""
