"""bench.py's N-GPU runs are replicas (the path shards no data): every rank times its own copy and the line
reports the slowest rank's time, with the whole job's throughput world x steps over it.  Two gloo ranks on the
CPU check that reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        out[rank] = bench.replica_rate(100.0 + 50.0 * rank, 10, device="cpu")
    finally:
        dist.destroy_process_group()


def test_replica_rate_takes_the_slowest_rank():
    import bench

    assert bench.replica_rate(200.0, 10, device="cpu") == (200.0, 50.0)  # one process: its own time
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
        got = dict(out)
    for r in range(world):
        ms, rate = got[r]
        assert ms == 150.0 and rate == pytest.approx(world * 10 / 0.150)
