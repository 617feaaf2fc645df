"""GPU: the reference tests' own sweep, case for case, against the oracle.

test_kronmult6_batched.cpp:443-477 (and the pbatched / xbatched tests) run
d = 1..6 x batch {1, 16, 128} x n {1, 2, 3, 4} on closed-form inputs
(test_kronmult6_batched.cpp:124-150); pbatched sends every output to column
1 (use_overlap_in_Y, test_kronmult6_pbatched.cpp:62), xbatched uses
lda = n + 3 (test_kronmult6_xbatched.cpp:65) and also runs in float
(:728-734).  Here each case runs through the library's C ABI and is compared
with the oracle: FP64 normwise relative error <= 1e-13 (the reference's own
bound is 1e-6 absolute), FP32 <= 1e-5."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden.make_golden import closed_form_batched
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

BATCHES = (1, 16, 128)
NS = (1, 2, 3, 4)


def _oracle_pointers(d, n, batch, A, lda, X, Yref, ycols):
    L = n ** d
    ap = [A.ctypes.data + 8 * (l * lda * n + k * lda * n * d) for k in range(batch)
          for l in range(d)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * L * c for c in ycols]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [lda] * d, xp, yp)


@pytest.mark.parametrize("d", range(1, 7))
def test_batched_sweep(gpu_lib, d):
    for batch in BATCHES:
        for n in NS:
            A, X = closed_form_batched(d, n, batch)
            Yref = np.zeros(n ** d * batch)
            oracle.kronmult_batched(d, n, A, X, Yref)
            dY = dev(np.zeros(n ** d * batch))
            need = kb.lib().kron_batched_workspace_bytes(d, n, batch)
            W = dev(np.zeros(max(1, need // 8))) if need else None
            kb.kronmult_batched(d, n, dev(A), dev(X), dY, W)
            assert rel_err(host(dY), Yref) <= 1e-13, (d, n, batch)


@pytest.mark.parametrize("d", range(1, 7))
def test_batched_sweep_fp32(gpu_lib, d):
    import torch

    for batch in BATCHES:
        for n in NS:
            A, X = closed_form_batched(d, n, batch)
            Yref = np.zeros(n ** d * batch)
            oracle.kronmult_batched(d, n, A, X, Yref)
            dY = torch.zeros(n ** d * batch, dtype=torch.float32, device="cuda")
            kb.kronmult_batched_f32(d, n, dev(A, torch.float32), dev(X, torch.float32), dY, None)
            assert rel_err(host(dY).astype(np.float64), Yref) <= 1e-5, (d, n, batch)


@pytest.mark.parametrize("d", range(1, 7))
def test_pbatched_sweep_all_outputs_in_column_one(gpu_lib, d):
    for batch in BATCHES:
        for n in NS:
            L = n ** d
            A, X = closed_form_batched(d, n, batch)
            Yref = np.zeros(L)
            _oracle_pointers(d, n, batch, A, n, X, Yref, [0] * batch)
            dA, dX, dY = dev(A), dev(X), dev(np.zeros(L))
            pX = ptrs(dX, [L * k for k in range(batch)])
            pY = ptrs(dY, [0] * batch)
            kb.kronmult_pbatched(d, n, dA, pX, pY)
            assert rel_err(host(dY), Yref) <= 1e-13, (d, n, batch)


@pytest.mark.parametrize("d", range(1, 7))
def test_xbatched_sweep_lda_n_plus_3(gpu_lib, d):
    for batch in BATCHES:
        for n in NS:
            L, lda = n ** d, n + 3
            A, X = closed_form_batched(d, n, batch, lda=lda)
            Yref = np.zeros(L)
            _oracle_pointers(d, n, batch, A, lda, X, Yref, [0] * batch)
            dA, dX, dY = dev(A), dev(X), dev(np.zeros(L))
            pA = ptrs(dA, [l * lda * n + k * lda * n * d for k in range(batch) for l in range(d)])
            pX = ptrs(dX, [L * k for k in range(batch)])
            pY = ptrs(dY, [0] * batch)
            kb.kronmult_xbatched(d, n, pA, lda, pX, pY)
            assert rel_err(host(dY), Yref) <= 1e-13, (d, n, batch)
            Xs = host(dX)
            assert np.array_equal(Xs, X), "X is never modified"
