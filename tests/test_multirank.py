"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): each rank
builds its own independently seeded mock (weak scaling, no collective on the
data path) and the timing / tuple totals are combined as the max and the sum
over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    cat, w, sp = bench.make_catalogue(bench.WORKLOAD, 0.001, bench.rank_seed(rank))
    t = bench.reduce_over_ranks(10.0 + rank, "max", "cpu")
    c = bench.reduce_over_ranks(cat.n, "sum", "cpu")
    out[rank] = (t, c, cat.n, float(cat.xyz[0, 0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0
    assert res[0][1] == res[1][1] == res[0][2] + res[1][2]
    # independent mocks
    assert res[0][3] != res[1][3]
