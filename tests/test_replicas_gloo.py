"""The multi-GPU path of this hot path is replicas only (no data-path
collective): one process per GPU, a barrier and the max over ranks of the
timed duration.  These run that host logic as world_size-2 gloo process
groups on the CPU, including the reference arm's rank-0-only behaviour."""
import io
import os
import sys
import contextlib

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, times, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.join(REPO, "lqcd-dwf-hmc_b200"))
    from b200dwf import replicas
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        replicas.barrier(dist)
        t = replicas.max_over_ranks(times[rank], dist)
        rate = replicas.whole_job_rate(1000.0, t, world)
        replicas.barrier(dist)
        out.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_max_over_ranks_and_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    times = [0.25, 0.40]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in res:
        assert t == pytest.approx(0.40)                 # every rank sees the slowest
        assert rate == pytest.approx(2 * 1000.0 / 0.40)  # whole-job units / slowest time


def test_single_process_needs_no_group():
    sys.path.insert(0, os.path.join(REPO, "lqcd-dwf-hmc_b200"))
    from b200dwf import replicas
    assert replicas.max_over_ranks(0.5, None) == 0.5
    assert replicas.whole_job_rate(10.0, 0.5, 1) == 20.0
    with pytest.raises(ValueError):
        replicas.whole_job_rate(1.0, 0.0, 1)


def test_reference_arm_prints_on_rank_zero_only():
    sys.path.insert(0, REPO)
    import bench

    class A:
        lattice = [4, 4, 4, 8]
        steps = 1
        warmup = 1
        gpus = 2

    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.reference_arm(A(), 1, 2)
    assert buf.getvalue() == ""
