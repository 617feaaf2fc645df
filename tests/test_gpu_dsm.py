"""GPU: FP64 d = 6, n = 6 with the intermediate kept in the cluster's shared
memory (two blocks per entry, no workspace) against the oracle.  That form
runs when the caller passes no W: batched calls, pointer layouts with
aliasing outputs, y only 8-byte aligned (element-wise red.add instead of the
bulk reduce-add), factors with lda > n; and, forced through the tuning
table, it agrees with the workspace form on the same inputs."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
D, N = 6, 6
L = N ** D


@pytest.fixture(autouse=True)
def _clean_table():
    kb.tune_clear()
    yield
    kb.tune_clear()


def test_batched_without_workspace(gpu_lib):
    batch = 5
    rng = np.random.default_rng(606)
    A = rng.standard_normal(N * N * D * batch) / np.sqrt(N)
    X = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * batch)
    Yref = Y0.copy()
    oracle.kronmult_batched(D, N, A, X, Yref)
    dY = dev(Y0)
    kb.kronmult_batched(D, N, dev(A), dev(X), dY, None)
    assert rel_err(host(dY), Yref) <= TOL64
    assert kb.lib().kron_device_status(1) == 0


@pytest.mark.parametrize("yshift", [0, 1])
def test_xbatched_aliasing_lda(gpu_lib, yshift):
    """Outputs aliased in pairs (atomic accumulation), A_l with lda = n + 1;
    yshift = 1 puts every y one element past a 16-byte boundary."""
    import torch

    batch, lda = 7, N + 1
    rng = np.random.default_rng(616 + yshift)
    Ap = rng.standard_normal(lda * N * D * batch) / np.sqrt(N)
    X = rng.uniform(-1, 1, L * batch)
    ny = (batch + 1) // 2
    Y0 = rng.uniform(-1, 1, L * ny + yshift)
    Yref = Y0.copy()
    ap = [Ap.ctypes.data + 8 * (k * D + l) * lda * N for k in range(batch) for l in range(D)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * (yshift + L * (k // 2)) for k in range(batch)]
    oracle.kronmult_general(D, [N] * D, [N] * D, ap, [lda] * D, xp, yp)
    dA, dX, dY = dev(Ap), dev(X), dev(Y0)
    pA = ptrs(dA, [(k * D + l) * lda * N for k in range(batch) for l in range(D)])
    pX = ptrs(dX, [L * k for k in range(batch)])
    pY = ptrs(dY, [yshift + L * (k // 2) for k in range(batch)])
    kb.kronmult_xbatched(D, N, pA, lda, pX, pY)
    torch.cuda.synchronize()
    assert rel_err(host(dY), Yref) <= TOL64
    assert kb.lib().kron_device_status(1) == 0


def test_shared_memory_and_workspace_forms_agree(gpu_lib):
    import torch

    batch = 4
    rng = np.random.default_rng(626)
    A = dev(rng.standard_normal(N * N * D * batch) / np.sqrt(N))
    X = dev(rng.uniform(-1, 1, L * batch))
    W = torch.empty(L * batch, dtype=torch.float64, device="cuda")
    Y1 = torch.zeros(L * batch, dtype=torch.float64, device="cuda")
    Y2 = torch.zeros_like(Y1)
    kb.kronmult_batched(D, N, A, X, Y1, W)
    kb.tune_set(D, N, "f64", "big", kb.BIG_SMEM_W)
    kb.kronmult_batched(D, N, A, X, Y2, W)
    torch.cuda.synchronize()
    assert rel_err(host(Y2), host(Y1)) <= TOL64
