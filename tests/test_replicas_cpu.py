"""The multi-GPU path is replicas only (no data-path collective): each rank
renders its own frames and the job's time is the slowest rank's.  Checked
here with 2 gloo ranks on the CPU, through bench.py's own helpers."""
import os
import socket
import sys

import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, ".."))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = [120.0, 180.0][rank]  # the ranks' own timed regions
        ms_max = bench.max_over_ranks(ms, world, device="cpu")
        value = bench.replica_rate(1920 * 1080, 10, ms_max, world)
        out.put((rank, ms_max, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = 2 * 1920 * 1080 * 10 / 0.180 / 1e6
    for rank, ms_max, value in results:
        assert ms_max == 180.0
        assert abs(value - want) < 1e-9 * want


def test_reference_arm_other_ranks_do_no_work(capsys):
    """Under torchrun only rank 0 runs the reference's CPU path and prints."""
    import argparse

    import bench

    args = argparse.Namespace(workload="forest", width=0, height=0, steps=1, warmup=0, gpus=2, views=64, scenes=16)
    bench.run_reference(args, rank=1)
    assert capsys.readouterr().out == ""
