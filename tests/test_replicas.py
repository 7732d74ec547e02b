"""The multi-GPU form of the path: independent replicas, throughput = all ranks' bytes over the
slowest rank's time.  Run here as two gloo ranks on the CPU (no GPU, no data-path collective)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        from falcons_b200 import replicas
        # rank r processed (r + 1) GB in (10 + 5 r) ms
        gbs, ms, total = replicas.job_throughput((rank + 1) * 1e9, 10.0 + 5.0 * rank)
        s = replicas.job_sum(rank + 1)
        out.put((rank, gbs, ms, total, s))
    finally:
        dist.destroy_process_group()


def test_job_throughput_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gbs, ms, total, s in res:
        assert ms == pytest.approx(15.0)          # the slowest rank's time
        assert total == pytest.approx(3e9)        # all ranks' bytes
        assert gbs == pytest.approx(3e9 / 0.015 / 1e9)
        assert s == pytest.approx(3.0)


def test_job_throughput_single_process():
    from falcons_b200 import replicas
    gbs, ms, total = replicas.job_throughput(2e9, 20.0)
    assert (gbs, ms, total) == (pytest.approx(100.0), 20.0, 2e9)
    assert replicas.job_sum(4.0) == 4.0
