"""The bench's multi-rank timing on CPU: with two gloo ranks, every rank gets
each value's maximum over the ranks (the whole job's time per step is its
slowest replica's), as `bench.py --gpus N` does over NCCL."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime
    import torch.distributed as tdist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.25], "cpu")
    finally:
        tdist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        got = dict(out)
    assert got == {0: [2.0, 10.0, 0.25], 1: [2.0, 10.0, 0.25]}
