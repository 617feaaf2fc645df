"""GPU: repeated application on a stream whose factors are kept in L2 gives
the oracle's result; the window is cleared afterwards."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu


def test_repeated_apply_with_persisting_factors(gpu_lib):
    import torch

    d, n, batch = 6, 4, 300
    L = n ** d
    rng = np.random.default_rng(77)
    A = rng.uniform(-1, 1, n * n * d * batch)
    X1 = rng.uniform(-1, 1, L * batch)
    X2 = rng.uniform(-1, 1, L * batch)
    Yref = np.zeros(L * batch)
    oracle.kronmult_batched(d, n, A, X1, Yref)
    oracle.kronmult_batched(d, n, A, X2, Yref)
    s = torch.cuda.Stream()
    dA = dev(A)
    dY = torch.zeros(L * batch, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(s):
        kb.l2_persist(dA, stream=s)
        kb.kronmult_batched(d, n, dA, dev(X1), dY, stream=s)
        kb.kronmult_batched(d, n, dA, dev(X2), dY, stream=s)
        kb.l2_persist_reset(stream=s)
    s.synchronize()
    assert rel_err(host(dY), Yref) <= 1e-13
