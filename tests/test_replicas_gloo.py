"""The multi-GPU mode of bench.py is N independent replicas (no collective on
the data path): ranks are timed between barriers and the job time is the max
over ranks. This runs that aggregation with 2 gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    ms = 10.0 * (rank + 1)  # rank 1 is the slow one
    job_ms = bench.max_over_ranks(ms, dist)
    dist.barrier()
    value = bench.job_value(world, 1000, 5, job_ms)
    with open(os.path.join(out_dir, f"r{rank}"), "w") as fh:
        fh.write(f"{job_ms} {value}")
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        job_ms, value = map(float, (tmp_path / f"r{r}").read_text().split())
        assert job_ms == 20.0  # every rank sees the max
        assert abs(value - 2 * 1000 * 5 / 0.020 / 1e6) < 1e-12
    del torch


def test_single_rank_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, None) == 12.5
    assert bench.job_value(1, 10_000_000, 100, 460.0) == pytest.approx(2173.913, rel=1e-6)
