"""The replica (N > 1) path of bench.py on CPU: two gloo ranks reduce their
times (max) and work (sum) the way the GPU ranks do, and each rank draws its
own seeded sweep.  No GPU."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    specs = bench.specs_for(rank)
    cells = sum(s["nx"] * s["nv"] for s in specs)
    maxes, sums = bench.reduce_over_ranks([1.0 + rank, 10.0 - rank], [cells], torch.device("cpu"))
    out[rank] = (maxes, sums, cells, len(specs))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_times_and_work():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    cells = [res[r][2] for r in range(world)]
    for r in range(world):
        maxes, sums, _, n = res[r]
        assert maxes == [2.0, 10.0]
        assert sums == [float(sum(cells))]
        assert n == 256
    assert cells[0] != cells[1]   # independent seeded sweeps per rank
