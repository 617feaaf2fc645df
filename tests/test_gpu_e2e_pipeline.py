"""GPU: the chunked end-to-end step of bench.py (host buffers up, one
library call per chunk, Y down, overlapped on three streams) returns the
oracle's result."""
import numpy as np
import pytest

import oracle
from tests.golden_cases import rel_err

pytestmark = pytest.mark.gpu


def test_batched_square_pipelined_e2e(gpu_lib):
    import torch

    import bench
    import kronmult_b200 as kb

    wl = bench.BatchedSquare(d=4, n=3, batch=43, seed=11)
    wl.setup(torch, kb, "atomic")
    wl.e2e_step()
    torch.cuda.synchronize()
    Yref = np.zeros(wl.L * wl.batch)
    oracle.kronmult_batched(wl.d, wl.n, wl.A, wl.X, Yref)
    assert rel_err(wl.hYout.numpy(), Yref) <= 1e-13


def test_xbatched_overlap_pipelined_e2e(gpu_lib):
    import torch

    import bench
    import kronmult_b200 as kb

    wl = bench.XbatchedOverlap(nelem=64, ncoup=4, seed=12)
    wl.setup(torch, kb, "atomic")
    wl.e2e_step()
    torch.cuda.synchronize()
    L, d, n = wl.L, wl.d, wl.n
    Yref = np.zeros(L * wl.nelem)
    X = wl.X.copy()
    ap = (wl.Apool.ctypes.data + 8 * wl.a_offsets()).tolist()
    xp = (X.ctypes.data + 8 * L * wl.xlist).tolist()
    yp = (Yref.ctypes.data + 8 * L * wl.ylist).tolist()
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
    assert rel_err(wl.hYout.numpy(), Yref) <= 1e-13
