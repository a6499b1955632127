"""Replicas on several GPUs: the only collective is the max over ranks of the
device-timed duration; the whole-job rate is all ranks' work over it.
Checked with two gloo ranks on the CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from cturbobfm_b200.replicas import max_over_ranks, whole_job_rate

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [10.0, 12.5][rank]
    mx = max_over_ranks(ms)
    rate = whole_job_rate(1000.0, world, mx)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mx, rate))


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, mx, rate in out:
        assert mx == 12.5
        assert rate == pytest.approx(2 * 1000.0 / 0.0125)


def test_single_process_needs_no_group():
    from cturbobfm_b200.replicas import max_over_ranks, whole_job_rate

    assert max_over_ranks(3.0) == 3.0
    assert whole_job_rate(10.0, 1, 1000.0) == 10.0
    with pytest.raises(ValueError):
        whole_job_rate(1.0, 1, 0.0)
