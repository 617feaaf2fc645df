"""GPU: pointer arrays built on the device from integer lists, and an
overlapping-output xbatched product through them against the oracle."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu


def test_pointers_from_lists_and_product(gpu_lib):
    import torch

    d, n, nelem, ncoup, npool = 3, 4, 64, 4, 5
    L = n ** d
    rng = np.random.default_rng(31)
    ylist = np.repeat(np.arange(nelem), ncoup).astype(np.int32)
    xlist = rng.integers(0, nelem, size=nelem * ncoup).astype(np.int32)
    aidx = rng.integers(0, npool, size=(nelem * ncoup, d))
    alist = (np.arange(d)[None, :] * npool + aidx).reshape(-1).astype(np.int32)
    Apool = rng.standard_normal(n * n * npool * d)
    X = rng.uniform(-1, 1, L * nelem)
    dA, dX = dev(Apool), dev(X)
    dY = torch.zeros(L * nelem, dtype=torch.float64, device="cuda")
    pA, pX, pY = kb.build_pointers(d, dA, n * n, dev(alist), dX, L, dev(xlist), dY, L,
                                   dev(ylist))
    assert np.array_equal(host(pA), dA.data_ptr() + 8 * n * n * alist.astype(np.int64))
    assert np.array_equal(host(pX), dX.data_ptr() + 8 * L * xlist.astype(np.int64))
    assert np.array_equal(host(pY), dY.data_ptr() + 8 * L * ylist.astype(np.int64))
    kb.kronmult_xbatched(d, n, pA, n, pX, pY)
    Yref = np.zeros(L * nelem)
    ap = (Apool.ctypes.data + 8 * n * n * alist.astype(np.int64)).tolist()
    xp = (X.ctypes.data + 8 * L * xlist.astype(np.int64)).tolist()
    yp = (Yref.ctypes.data + 8 * L * ylist.astype(np.int64)).tolist()
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
    assert rel_err(host(dY), Yref) <= 1e-13


def test_identity_lists(gpu_lib):
    import torch

    d, batch, L = 2, 1000, 9
    A = torch.zeros(d * batch * 9, dtype=torch.float64, device="cuda")
    X = torch.zeros(L * batch, dtype=torch.float64, device="cuda")
    Y = torch.zeros(L * batch, dtype=torch.float64, device="cuda")
    pA = torch.empty(batch * d, dtype=torch.int64, device="cuda")
    pX = torch.empty(batch, dtype=torch.int64, device="cuda")
    rc = kb.lib().kron_build_pointers_async(d, batch, A.data_ptr(), 9, None, X.data_ptr(), L,
                                            None, Y.data_ptr(), L, None, pA.data_ptr(),
                                            pX.data_ptr(), None, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(host(pA), A.data_ptr() + 8 * 9 * np.arange(batch * d))
    assert np.array_equal(host(pX), X.data_ptr() + 8 * L * np.arange(batch))
