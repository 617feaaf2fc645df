"""GPU: kgemm_{nn,nt,tt}_batched over a sample of the reference tests' sweep
(test_kgemm_nn_batched.cpp:491-533: mm, nn, kk from 1 to 64, batch 1..15)
with per-entry leading dimensions, against the oracle's naive product.
alpha/beta cover the tests' (1.3, 1.2), the atomic branch beta == 1 (which
the reference tests never reach) including every C aliasing one matrix, and
beta == 0 (C never read)."""
import itertools

import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

SIZES = (1, 8, 29, 64)


def _case(op, mm, nn, kk, batch, alpha, beta, alias, rng):
    import torch

    rA = kk if op == "tt" else mm
    cA = mm if op == "tt" else kk
    rB = kk if op == "nn" else nn
    cB = nn if op == "nn" else kk
    ldA = rA + rng.integers(0, 3, size=batch)
    ldB = rB + rng.integers(0, 3, size=batch)
    ldC = mm + rng.integers(0, 3, size=batch)
    offA = np.concatenate([[0], np.cumsum(ldA * cA)])
    offB = np.concatenate([[0], np.cumsum(ldB * cB)])
    offC = np.concatenate([[0], np.cumsum(ldC * nn)])
    if alias:
        ldC[:] = ldC[0]
        offC = np.zeros(batch + 1, dtype=np.int64)
        offC[1:] = 0
        csize = int(ldC[0] * nn)
    else:
        csize = int(offC[-1])
    A = rng.uniform(-1, 1, int(offA[-1]))
    B = rng.uniform(-1, 1, int(offB[-1]))
    C0 = rng.uniform(-1, 1, max(csize, 1))
    Cref = C0.copy()
    oracle.kgemm_batched(op, mm, nn, kk, alpha,
                         [A.ctypes.data + 8 * int(offA[b]) for b in range(batch)], ldA.tolist(),
                         [B.ctypes.data + 8 * int(offB[b]) for b in range(batch)], ldB.tolist(),
                         beta, [Cref.ctypes.data + 8 * int(offC[b]) for b in range(batch)],
                         ldC.tolist())
    dA, dB, dC = dev(A), dev(B), dev(C0)
    li = lambda v: torch.tensor(v, dtype=torch.int32, device="cuda")  # noqa: E731
    kb.kgemm_batched(op, mm, nn, kk, alpha, ptrs(dA, offA[:-1]), li(ldA), ptrs(dB, offB[:-1]),
                     li(ldB), beta, ptrs(dC, offC[:-1]), li(ldC))
    return rel_err(host(dC), Cref)


@pytest.mark.parametrize("op", ["nn", "nt", "tt"])
def test_kgemm_sweep(gpu_lib, op):
    rng = np.random.default_rng({"nn": 11, "nt": 12, "tt": 13}[op])
    for mm, nn, kk in itertools.product(SIZES, SIZES, SIZES):
        for batch in (1, 15):
            for alpha, beta in ((1.3, 1.2), (1.0, 1.0), (0.7, 0.0)):
                err = _case(op, mm, nn, kk, batch, alpha, beta, False, rng)
                assert err <= 1e-13, (op, mm, nn, kk, batch, alpha, beta, err)


@pytest.mark.parametrize("op", ["nn", "nt", "tt"])
def test_kgemm_beta_one_aliasing_outputs(gpu_lib, op):
    """beta == 1 accumulates atomically: fifteen products into one C."""
    rng = np.random.default_rng(21)
    for mm, nn, kk in ((8, 8, 8), (29, 64, 8), (64, 1, 29)):
        err = _case(op, mm, nn, kk, 15, 1.1, 1.0, True, rng)
        assert err <= 1e-13, (op, mm, nn, kk, err)


@pytest.mark.parametrize("op", ["nn", "nt", "tt"])
def test_kgemm_tile_kernel_sizes(gpu_lib, op):
    """Entries beyond 64 x 64 x 64 take the CUDA-core tile kernel; entries up
    to it take the tensor-core kernel unless KRON_KGEMM_CUDA_CORES is set,
    which runs the tile kernel on them too.  Both against the oracle."""
    import os

    rng = np.random.default_rng({"nn": 31, "nt": 32, "tt": 33}[op])
    for mm, nn, kk in ((65, 64, 64), (64, 70, 3), (9, 8, 130)):
        for alpha, beta in ((1.3, 1.2), (1.0, 1.0)):
            err = _case(op, mm, nn, kk, 5, alpha, beta, False, rng)
            assert err <= 1e-13, (op, mm, nn, kk, alpha, beta, err)
    os.environ["KRON_KGEMM_CUDA_CORES"] = "1"
    try:
        for mm, nn, kk in ((64, 64, 64), (29, 8, 1)):
            err = _case(op, mm, nn, kk, 7, 1.3, 1.2, False, rng)
            assert err <= 1e-13, (op, mm, nn, kk, err)
    finally:
        del os.environ["KRON_KGEMM_CUDA_CORES"]
