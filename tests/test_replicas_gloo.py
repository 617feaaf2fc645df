"""The multi-GPU path of bench.py is replicas only: every rank runs the whole
workload on its own GPU, no collective touches the data, and the timed
numbers are the max over ranks.  Here the max-over-ranks reduction and the
launcher's environment parsing run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    w, r, local = bench.dist_setup()
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r reports step time 10 + r ms and e2e time 50 - r ms
        out[rank] = (w, r, local, bench.max_over_ranks(dist, [10.0 + rank, 50.0 - rank], "cpu"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        w, r, local, vals = res[rank]
        assert (w, r, local) == (world, rank, rank)
        assert vals == [10.0 + world - 1, 50.0]


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(None, [3, 4.5], "cpu") == [3.0, 4.5]
