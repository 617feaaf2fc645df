"""Owner-computes sharding on the CPU: kron_owner_partition through the C ABI
(host function, no GPU) and the exchange of owned output ranges between two
gloo ranks.

The partition must give every entry to exactly one rank, give each rank one
contiguous range of output columns covering every output its entries write
(so no output is touched by two ranks), list a rank's entries by increasing
output with the batch order kept inside one output, and balance entry counts
to within one output group.  In the two-rank test each rank computes its
share with the oracle standing in for its GPU, the ranks exchange their owned
columns with OwnerShard.gather, and both must end with the whole batch's
result."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import kronmult_b200 as kb
from kronmult_b200.owner import OwnerShard, owner_partition

KRON_ERROR_INVALID_VALUE = 1


def _check_partition(y, nranks):
    order, eb, ob = owner_partition(y, nranks)
    B = y.size
    assert sorted(order.tolist()) == list(range(B))
    assert eb[0] == 0 and eb[-1] == B and np.all(np.diff(eb) >= 0)
    assert ob[0] == 0 and np.all(np.diff(ob) >= 0)
    assert ob[-1] == (y.max() + 1 if B else 0)
    ys = y[order]
    # increasing outputs, batch order inside one output (stable)
    assert np.all(np.diff(ys) >= 0)
    for v in np.unique(ys):
        idx = order[ys == v]
        assert np.all(np.diff(idx) > 0)
    for r in range(nranks):
        mine = order[eb[r]:eb[r + 1]]
        assert np.all((y[mine] >= ob[r]) & (y[mine] < ob[r + 1]))
    # an output group never straddles two ranks, and each cut is the group
    # start nearest its target, so a rank's count is off by < one group
    if B:
        big = np.bincount(y).max()
        for r in range(nranks):
            assert abs(int(eb[r + 1] - eb[r]) - B / nranks) <= big + 1
    return order, eb, ob


@pytest.mark.parametrize("seed,B,ny,nranks", [
    (0, 1, 1, 1), (1, 10, 4, 3), (2, 1000, 97, 4), (3, 131072, 8192, 8),
    (4, 500, 3, 8), (5, 64, 64, 2), (6, 7, 1000000, 3),
])
def test_partition_properties(seed, B, ny, nranks):
    y = np.random.default_rng(seed).integers(0, ny, size=B).astype(np.int32)
    _check_partition(y, nranks)


def test_partition_of_the_coupled_grid():
    # the overlapping-output workload: 8192 elements x 16 couplings, entries
    # grouped by output element; 8 ranks get 16384 entries each
    y = np.repeat(np.arange(8192, dtype=np.int32), 16)
    order, eb, ob = _check_partition(y, 8)
    assert np.all(np.diff(eb) == 16384)
    assert np.all(np.diff(ob) == 1024)


def test_partition_edge_cases():
    order, eb, ob = owner_partition(np.zeros(0, np.int32), 3)
    assert eb.tolist() == [0, 0, 0, 0] and ob.tolist() == [0, 0, 0, 0]
    # one output for everything: one rank takes it all
    order, eb, ob = _check_partition(np.full(9, 5, np.int32), 4)
    assert sorted(np.diff(eb).tolist()) == [0, 0, 0, 9]


def test_partition_rejects_bad_arguments():
    lib = kb.lib()
    y = np.array([0, -1, 2], dtype=np.int32)
    out = np.empty(3, np.int32)
    b = np.empty(3, np.int32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert lib.kron_owner_partition(3, p(y), 2, p(out), p(b), p(b)) == KRON_ERROR_INVALID_VALUE
    y[1] = 1
    assert lib.kron_owner_partition(3, p(y), 0, p(out), p(b), p(b)) == KRON_ERROR_INVALID_VALUE
    assert lib.kron_owner_partition(-1, p(y), 2, p(out), p(b), p(b)) == KRON_ERROR_INVALID_VALUE
    assert lib.kron_owner_partition(3, None, 2, p(out), p(b), p(b)) == KRON_ERROR_INVALID_VALUE
    assert lib.kron_owner_partition(3, p(y), 2, p(out), None, p(b)) == KRON_ERROR_INVALID_VALUE


# ---------------------------------------------------------------- two gloo ranks
D, N, NEL, NPOOL = 3, 3, 40, 5
L = N ** D


def _problem():
    rng = np.random.default_rng(99)
    nent = 150
    ylist = rng.integers(0, NEL, size=nent).astype(np.int32)
    xlist = rng.integers(0, NEL, size=nent).astype(np.int32)
    alist = rng.integers(0, NPOOL * D, size=nent * D).astype(np.int32)
    Apool = rng.standard_normal(N * N * NPOOL * D)
    X = rng.uniform(-1, 1, L * NEL)
    return ylist, xlist, alist, Apool, X


def _oracle(entries, ylist, xlist, alist, Apool, X, Y):
    """The entries in list order: one oracle thread, so entries that share
    an output add up in that order (bit-reproducible)."""
    import oracle

    if len(entries) == 0:
        return
    old = oracle.num_threads()
    oracle.set_threads(1)
    ap = [Apool.ctypes.data + 8 * N * N * int(alist[D * k + l]) for k in entries
          for l in range(D)]
    oracle.kronmult_general(D, [N] * D, [N] * D, ap, [N] * D,
                            [X.ctypes.data + 8 * L * int(xlist[k]) for k in entries],
                            [Y.ctypes.data + 8 * L * int(ylist[k]) for k in entries])
    oracle.set_threads(old)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ylist, xlist, alist, Apool, X = _problem()
        sh = OwnerShard(D, xlist, ylist, alist, rank, world)
        Y = np.zeros(L * NEL)
        # the oracle stands in for this rank's GPU: its entries only
        _oracle(sh.entries, ylist, xlist, alist, Apool, X, Y)
        touched = np.flatnonzero(Y.reshape(NEL, L).any(axis=1))
        own = bool(np.all((touched >= sh.out_lo) & (touched < sh.out_hi)))
        Yt = torch.from_numpy(Y)
        sh.gather(Yt, L)
        out[rank] = (own, len(sh), Yt.numpy().copy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_exchange_owned_outputs():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    ylist, xlist, alist, Apool, X = _problem()
    # the whole batch in the partition's order (each output summed in batch order)
    order, _, _ = owner_partition(ylist, 1)
    expect = np.zeros(L * NEL)
    _oracle(order, ylist, xlist, alist, Apool, X, expect)
    assert res[0][1] + res[1][1] == ylist.size
    for r in range(world):
        own, cnt, Y = res[r]
        assert own, f"rank {r} wrote outside its output range"
        # every output column was summed by one rank in batch order: bitwise
        assert np.array_equal(Y, expect)
