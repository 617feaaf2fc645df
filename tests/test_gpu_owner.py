"""Owner-computes sharding on the GPU: each rank's share (OwnerShard.apply:
pointer arrays built on the device from the index lists, one xbatched call)
run through the CUDA library, checked against the oracle.

This run has one GPU, so the ranks run one after another on it, each into
its own copy of Y; their kernels never wait on one another, so this is the
same work each GPU would do.  Every rank must leave the columns it does not
own untouched, the owned ranges put together must equal the whole batch's
result (FP64 tolerance 1e-13 with atomic adds), and in the deterministic
mode they must equal, bit for bit, one segmented call over the whole batch
(each output is summed in batch order either way)."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from kronmult_b200.owner import OwnerShard
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu


def _problem(d, n, nel, nent, npool, seed):
    rng = np.random.default_rng(seed)
    L = n ** d
    ylist = rng.integers(0, nel, size=nent).astype(np.int32)
    xlist = rng.integers(0, nel, size=nent).astype(np.int32)
    alist = rng.integers(0, npool * d, size=nent * d).astype(np.int32)
    Apool = rng.standard_normal(n * n * npool * d) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * nel)
    Y0 = rng.uniform(-1, 1, L * nel)
    return ylist, xlist, alist, Apool, X, Y0


def _oracle(d, n, ylist, xlist, alist, Apool, X, Y):
    L = n ** d
    ap = [Apool.ctypes.data + 8 * n * n * int(a) for a in alist]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d,
                            [X.ctypes.data + 8 * L * int(j) for j in xlist],
                            [Y.ctypes.data + 8 * L * int(i) for i in ylist])


@pytest.mark.parametrize("d,n,nel,nent,nranks,deterministic", [
    (3, 8, 256, 2048, 3, False),   # the tensor-core n = 8 kernel
    (3, 8, 256, 2048, 4, True),
    (4, 5, 60, 700, 2, False),     # pipelined kernel
    (6, 4, 40, 300, 3, True),
    (2, 3, 9, 50, 8, False),       # more ranks than some outputs have entries
])
def test_owner_shards_match_the_whole_batch(gpu_lib, d, n, nel, nent, nranks, deterministic):
    import torch

    L = n ** d
    ylist, xlist, alist, Apool, X, Y0 = _problem(d, n, nel, nent, 8, 31 * d + n + nranks)
    expect = Y0.copy()
    _oracle(d, n, ylist, xlist, alist, Apool, X, expect)
    dA, dX = dev(Apool), dev(X)
    assembled = np.empty_like(Y0)
    counts = 0
    for r in range(nranks):
        sh = OwnerShard(d, xlist, ylist, alist, r, nranks)
        counts += len(sh)
        dY = dev(Y0)
        sh.apply(n, dA, n * n, n, dX, L, dY, L, deterministic=deterministic)
        got = host(dY)
        lo, hi = sh.out_lo * L, sh.out_hi * L
        # columns outside the owned range are untouched
        assert np.array_equal(got[:lo], Y0[:lo]) and np.array_equal(got[hi:], Y0[hi:])
        assembled[lo:hi] = got[lo:hi]
    assembled[sh.out_bounds[-1] * L:] = Y0[sh.out_bounds[-1] * L:]
    assert counts == nent
    assert rel_err(assembled, expect) <= 1e-13
    assert gpu_lib.kron_device_status(1) == 0

    if deterministic:
        # one segmented call over the whole batch sums each output in batch
        # order too: the shards reproduce it bit for bit
        dY = dev(Y0)
        pA, pX, pY = kb.build_pointers(d, dA, n * n, dev(alist), dX, L, dev(xlist), dY, L,
                                       dev(ylist))
        seg = kb.Segments(pY)
        kb.kronmult_xbatched_segmented(d, n, pA, n, pX, pY, seg)
        whole = host(dY)
        seg.close()
        assert np.array_equal(assembled, whole)
        torch.cuda.synchronize()
