"""The N > 1 bench path on CPU: independent replicas whose only collective is
the max-over-ranks timing and the summed point count (world size 2, gloo on
127.0.0.1), and the reference arm's non-zero ranks exiting without work."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: its own device time, end-to-end time and counted points
        out = bench.reduce_over_ranks(dist, "cpu", 1.0 + rank, 2.5 - rank, 3 + 4 * rank)
        q.put((rank, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_reduce_max_time_and_sum_points():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=10) for _ in procs)
    # every rank sees the same whole-job figures: max times, summed points
    assert got[0] == got[1] == (2.0, 2.5, 10)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), dict(workload="diode2d", small=True, steps=1, warmup=0, gpus=2))()
    assert bench.run_reference(args) is None
