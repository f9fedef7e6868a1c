"""The benchmark's replica mode (bench.py --gpus N: one process per GPU, each stepping its own
copy of the scene; no collective on the data path) on CPU: two gloo ranks with different
timings agree on the slowest rank's time, and the whole-job rate counts both ranks' steps."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        own = 100.0 + 25.0 * rank  # this rank's device time for its timed steps (ms)
        got = bench.slowest_ms(own, world, "cpu")
        with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{got!r} {bench.whole_job_rate(world, 20, got)!r}")
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank(tmp_path):
    world = 2
    port = _free_port()
    mp.start_processes(_rank, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn")
    for rank in range(world):
        ms, rate = map(float, (tmp_path / f"rank{rank}.txt").read_text().split())
        assert ms == 125.0
        assert rate == pytest.approx(2 * 20 / 0.125)


def test_single_rank_keeps_its_own_time():
    import bench
    assert bench.slowest_ms(42.0, 1, "cpu") == 42.0
    assert bench.whole_job_rate(1, 300, 1000.0) == pytest.approx(300.0)
