"""bench.py's multi-GPU path: independent replicas, the slowest rank's time,
whole-job throughput. Run as two gloo ranks on CPU (no GPU, no collective on
the data path)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        ms, e2e = bench.max_over_ranks([10.0 + 5.0 * rank, 1.0 + 0.5 * rank], ws, "cpu")
        out[rank] = (ms, e2e, *bench.replica_throughput(ws, 1000, 20, ms, e2e))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ws = 2
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(ws, _free_port(), out), nprocs=ws, start_method="spawn")
    assert out[0] == out[1]
    ms, e2e, value, e2e_value = out[0]
    assert (ms, e2e) == (15.0, 1.5)
    assert value == pytest.approx(2 * 1000 * 20 / 0.015)
    assert e2e_value == pytest.approx(2 * 1000 * 20 / 1.5)


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks([3.0, 4.0], 1, "cpu") == [3.0, 4.0]
