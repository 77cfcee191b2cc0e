"""The multi-GPU form of bench.py is replicas: every rank runs the same step
and the job's throughput is the sum of the ranks' bytes over the slowest
rank's time.  Checked here with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # rank r takes (r + 1) ms per step and moves 1e9 bytes per step
        gbs, ms_max = bench.job_throughput(float(rank + 1), 1e9, world)
        out[rank] = (gbs, ms_max)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # the slowest rank (2 ms) sets the pace; both ranks' bytes count
    for r in range(world):
        gbs, ms_max = out[r]
        assert ms_max == pytest.approx(2.0)
        assert gbs == pytest.approx(world * 1e9 / 2e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    gbs, ms = bench.job_throughput(4.0, 2e9, 1)
    assert ms == 4.0 and gbs == pytest.approx(500.0)


def test_reference_arm_other_ranks_do_nothing(capsys):
    # under torchrun only rank 0 times the reference's CPU path and prints
    sys.path.insert(0, ROOT)
    import bench
    bench.run_reference(None, 1, 2)
    assert capsys.readouterr().out == ""
