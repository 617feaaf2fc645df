"""GPU: the slab-cluster kernel (d = 6, n = 6; one cluster of twelve blocks
per entry holding half slabs, or six holding whole slabs; no workspace)
against the oracle, through the C ABI.

Covers every path of the kernel:
- both stages of each block's ring, with batches from 1 entry to several
  entries per cluster;
- the TMA copies and their plain-load fallbacks (x not 16-byte aligned;
  xbatched factors with lda > n);
- results added into y at any alignment (y shifted by one element);
- outputs that alias (pbatched);
- FP32 and FP64;
- the side kernel that takes a share of large FP64 batches on the SMs the
  clusters leave idle (batched and aliasing pbatched, with W).
FP64 bar: normwise relative error <= 1e-13; FP32 <= 1e-5 against the FP64
oracle."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

D, N = 6, 6
L = N ** D
TOL = {"f64": 1e-13, "f32": 1e-5}


@pytest.fixture(autouse=True)
def _clean_table():
    kb.tune_clear()
    yield
    kb.tune_clear()


def _inputs(batch, seed, ny=None):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal(N * N * D * batch) / np.sqrt(N)
    X = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * (ny or batch))
    return A, X, Y0


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("batch", [1, 7, 40, 150])
@pytest.mark.parametrize("forced", [None, 0, kb.SLAB_NO_ROTATE, kb.SLAB_WHOLE,
                                    kb.SLAB_WHOLE | kb.SLAB_NO_ROTATE, kb.SLAB_PLAIN_Y])
def test_slab_batched(gpu_lib, prec, batch, forced):
    """forced: None = built-in choice, else the slab variant with that param
    (half or whole slabs per block, with and without the lane rotation of
    the first pass, y by atomics or by loads and stores)."""
    import torch

    if forced is not None:
        kb.tune_set(D, N, prec, "slab", forced)
    A, X, Y0 = _inputs(batch, 600 + batch)
    Yref = Y0.copy()
    oracle.kronmult_batched(D, N, A, X, Yref)
    dt = torch.float64 if prec == "f64" else torch.float32
    dA, dX, dY = dev(A, dt), dev(X, dt), dev(Y0, dt)
    X0 = dX.clone()
    # no workspace: the slab kernel needs none
    if prec == "f64":
        kb.kronmult_batched(D, N, dA, dX, dY, None)
    else:
        kb.kronmult_batched_f32(D, N, dA, dX, dY, None)
    assert rel_err(host(dY).astype(np.float64), Yref) <= TOL[prec]
    assert torch.equal(dX, X0), "x must be preserved"
    assert kb.lib().kron_device_status(1) == 0


def test_slab_pbatched_aliasing(gpu_lib):
    """Outputs aliased in runs of three: the bulk reduce-adds of different
    clusters land on the same y."""
    batch = 61
    ny = (batch + 2) // 3
    A, X, Y0 = _inputs(batch, 611, ny)
    Yref = Y0.copy()
    ap = [A.ctypes.data + 8 * (k * D + l) * N * N for k in range(batch) for l in range(D)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * L * (k // 3) for k in range(batch)]
    oracle.kronmult_general(D, [N] * D, [N] * D, ap, [N] * D, xp, yp)
    dA, dX, dY = dev(A), dev(X), dev(Y0)
    pX = ptrs(dX, [L * k for k in range(batch)])
    pY = ptrs(dY, [L * (k // 3) for k in range(batch)])
    kb.kronmult_pbatched(D, N, dA, pX, pY)
    assert rel_err(host(dY), Yref) <= TOL["f64"]
    assert kb.lib().kron_device_status(1) == 0


@pytest.mark.parametrize("xoff,yoff", [(1, 0), (0, 1), (1, 1), (0, 0)])
def test_slab_xbatched_fallbacks(gpu_lib, xoff, yoff):
    """xbatched with lda = n + 2 (factors by plain loads), x and/or y shifted
    by one element off 16-byte alignment (slab by plain loads, results by
    atomic adds)."""
    batch, lda, npool = 23, N + 2, 5
    rng = np.random.default_rng(620 + xoff + 2 * yoff)
    Apool = rng.standard_normal(lda * N * npool * D) / np.sqrt(N)
    X = rng.uniform(-1, 1, L * batch + xoff)
    Y0 = rng.uniform(-1, 1, L * batch + yoff)
    aidx = rng.integers(0, npool, size=(batch, D))
    aoff = [lda * N * (l * npool + int(aidx[k, l])) for k in range(batch) for l in range(D)]
    Yref = Y0.copy()
    oracle.kronmult_general(D, [N] * D, [N] * D, [Apool.ctypes.data + 8 * o for o in aoff],
                            [lda] * D, [X.ctypes.data + 8 * (xoff + L * k) for k in range(batch)],
                            [Yref.ctypes.data + 8 * (yoff + L * k) for k in range(batch)])
    dAp, dX, dY = dev(Apool), dev(X), dev(Y0)
    pA = ptrs(dAp, aoff)
    pX = ptrs(dX, [xoff + L * k for k in range(batch)])
    pY = ptrs(dY, [yoff + L * k for k in range(batch)])
    kb.tune_set(D, N, "f64", "slab", 0)
    kb.kronmult_xbatched(D, N, pA, lda, pX, pY)
    assert rel_err(host(dY), Yref) <= TOL["f64"]
    assert kb.lib().kron_device_status(1) == 0


def test_slab_matches_two_phase(gpu_lib):
    """The slab kernel and the cluster two-phase kernel agree on the same
    batch (two independent kernels; both also checked against the oracle
    elsewhere)."""
    import torch

    batch = 33
    A, X, Y0 = _inputs(batch, 630)
    dA, dX = dev(A), dev(X)
    out = {}
    for v, q in (("slab", 0), ("big", 2)):
        kb.tune_set(D, N, "f64", v, q)
        dY = dev(Y0)
        W = torch.empty(L * batch, dtype=torch.float64, device="cuda")
        kb.kronmult_batched(D, N, dA, dX, dY, W)
        out[v] = host(dY)
    assert rel_err(out["slab"], out["big"]) <= 1e-14


@pytest.mark.parametrize("forced", [None, 0, kb.SLAB_NO_SIDE, kb.SLAB_WHOLE])
def test_slab_with_side_kernel(gpu_lib, forced):
    """FP64 batches of 512 entries or more with a workspace: a share of the
    entries runs concurrently on the cluster two-phase kernel (second
    stream) on the SMs the slab clusters leave idle.  Batched with W, the
    default and forced forms, and the opt-out bit."""
    import torch

    batch = 700
    if forced is not None:
        kb.tune_set(D, N, "f64", "slab", forced)
    A, X, Y0 = _inputs(batch, 6006)
    Yref = Y0.copy()
    oracle.kronmult_batched(D, N, A, X, Yref)
    dY = dev(Y0)
    W = torch.empty(L * batch, dtype=torch.float64, device="cuda")
    kb.kronmult_batched(D, N, dev(A), dev(X), dY, W)
    assert rel_err(host(dY), Yref) <= TOL["f64"]
    assert gpu_lib.kron_device_status(1) == 0


def test_slab_with_side_kernel_aliasing_pbatched(gpu_lib):
    """pbatched with outputs that alias (600 entries onto 150 columns) and a
    W pointer per entry: both kernels add into shared columns atomically."""
    import torch

    batch, ny = 600, 150
    A, X, Y0 = _inputs(batch, 6007, ny)
    yl = np.random.default_rng(6008).integers(0, ny, size=batch)
    Yref = Y0.copy()
    oracle.kronmult_general(D, [N] * D, [N] * D,
                            [A.ctypes.data + 8 * N * N * (D * k + l) for k in range(batch)
                             for l in range(D)],
                            [N] * D, [X.ctypes.data + 8 * L * k for k in range(batch)],
                            [Yref.ctypes.data + 8 * L * int(j) for j in yl])
    dX, dY = dev(X), dev(Y0)
    W = torch.empty(L * batch, dtype=torch.float64, device="cuda")
    kb.kronmult_pbatched(D, N, dev(A), ptrs(dX, L * np.arange(batch)), ptrs(dY, L * yl),
                         pW=ptrs(W, L * np.arange(batch)))
    assert rel_err(host(dY), Yref) <= TOL["f64"]
    assert gpu_lib.kron_device_status(1) == 0
