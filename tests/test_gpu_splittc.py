"""Split precision for d = 6, n = 8 on the tcgen05 tensor cores
(kron_splittc.cu): FP64 data, exact BF16 slice products, FP32 accumulators,
FP64 reconstruction.  Checked through the C ABI (kronmult_batched_split_async)
against the oracle at the split path's tolerance, 1e-12 normwise, with the
variant forced by the tuning table and as the built-in choice; the device
status word must stay 0.  Inputs include rows of mixed magnitude and exact
zeros (fibres whose scale exponent is 0)."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

TOL_SPLIT = 1e-12


@pytest.fixture(autouse=True)
def _clean_table():
    kb.tune_clear()
    yield
    kb.tune_clear()


@pytest.mark.parametrize("batch,forced,scaled", [
    (1, True, False), (3, True, True), (5, False, False), (9, False, True)])
def test_split_tc_matches_oracle(gpu_lib, batch, forced, scaled):
    import torch

    d, n = 6, 8
    L = n ** d
    rng = np.random.default_rng(600 + batch)
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * batch)
    if scaled:
        # fibres and factor rows spanning many binades, some exactly zero
        X *= np.exp2(rng.integers(-30, 30, size=X.size))
        X[rng.random(X.size) < 0.05] = 0.0
        A *= np.exp2(rng.integers(-10, 10, size=A.size))
        A[::17] = 0.0
    Y0 = rng.uniform(-1, 1, L * batch)
    expect = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, expect)
    if forced:
        kb.tune_set(d, n, "split", "split_tc")
    dY = dev(Y0)
    W = torch.empty(L * batch, dtype=torch.float64, device="cuda")
    kb.kronmult_batched_split(d, n, dev(A), dev(X), dY, W)
    got = host(dY)
    err = rel_err(got, expect)
    assert err <= TOL_SPLIT, err
    assert gpu_lib.kron_device_status(1) == 0
