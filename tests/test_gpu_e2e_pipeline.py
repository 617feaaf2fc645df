"""GPU: the end-to-end steps of bench.py (host buffers up, the library
call(s), Y down; chunked and overlapped on three streams for the batched and
atomic xbatched workloads) return the oracle's or the reference's result, for
every workload of the bench at small sizes."""
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


@pytest.mark.parametrize("n,batch,prec,tol", [
    (6, 24, "f64", 1e-13),     # slab-cluster kernel per chunk
    (6, 24, "f32", 1e-5),
    (6, 10, "split", 1e-12),   # two-phase launches through each chunk's W
    (8, 4, "split", 1e-12),    # tensor-core split, one entry per chunk
])
def test_batched_d6_pipelined_e2e(gpu_lib, n, batch, prec, tol):
    import torch

    import bench
    import kronmult_b200 as kb

    wl = bench.BatchedSquare(d=6, n=n, batch=batch, precision=prec, dist="normal", seed=13)
    wl.setup(torch, kb, "atomic")
    wl.e2e_step()
    torch.cuda.synchronize()
    Yref = np.zeros(wl.L * wl.batch)
    oracle.kronmult_batched(wl.d, wl.n, wl.A, wl.X, Yref)
    assert rel_err(wl.hYout.double().numpy(), Yref) <= tol
    assert kb.lib().kron_device_status(1) == 0


def test_uneven_batch_e2e(gpu_lib):
    """Host buffers up, one plan execution, Y down; against the reference's
    own per-entry output (its OpenMP build)."""
    import torch

    import bench
    import kronmult_b200 as kb

    wl = bench.UnevenBatch(nent=300, seed=14)
    wl.setup(torch, kb, "atomic")
    wl.e2e_step()
    torch.cuda.synchronize()
    assert rel_err(wl.hYout.numpy(), wl.reference_y()) <= 1e-13


def test_xbatched_big_e2e(gpu_lib):
    import torch

    import bench
    import kronmult_b200 as kb

    wl = bench.XbatchedBig(batch=8, nout=6)
    wl.setup(torch, kb, "atomic")
    wl.e2e_step()
    torch.cuda.synchronize()
    assert rel_err(wl.hYout.numpy(), wl.reference_y()) <= 1e-13


def test_kgemm_e2e(gpu_lib):
    """C_k += A_k B_k from host buffers: C0 plus the reference's product."""
    import torch

    import bench
    import kronmult_b200 as kb

    wl = bench.KgemmBatched(batch=64)
    wl.setup(torch, kb, "atomic")
    wl.e2e_step()
    torch.cuda.synchronize()
    assert rel_err(wl.hYout.numpy(), wl.C0 + wl.reference_y()) <= 1e-13
