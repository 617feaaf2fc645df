"""GPU: the autotuner's choices and every forced kernel variant against the
oracle (FP64 normwise relative error <= 1e-13, FP32 <= 1e-5).  Forcing a
variant through the choice table runs that kernel alone, so each variant's
parity is checked here, not only the one the built-in order prefers."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-13, "f32": 1e-5}


@pytest.fixture(autouse=True)
def _clean_table():
    kb.tune_clear()
    yield
    kb.tune_clear()


def _batched(d, n, batch, prec, seed, with_w=False):
    import torch

    rng = np.random.default_rng(seed)
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, n ** d * batch)
    Y0 = rng.uniform(-1, 1, n ** d * batch)
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    dt = torch.float64 if prec == "f64" else torch.float32
    dY = dev(Y0, dt)
    need = kb.lib().kron_batched_workspace_bytes(d, n, batch)
    if with_w:
        need = max(need, 8 * n ** d * batch)
    W = torch.empty(max(1, need // 8), dtype=dt, device="cuda") if need else None
    if prec == "f64":
        kb.kronmult_batched(d, n, dev(A), dev(X), dY, W)
    else:
        kb.kronmult_batched_f32(d, n, dev(A, dt), dev(X, dt), dY, W)
    err = rel_err(host(dY).astype(np.float64), Yref)
    assert err <= TOL[prec], err
    assert kb.lib().kron_device_status(1) == 0


@pytest.mark.parametrize("d,n,prec,batch", [
    (6, 4, "f64", 300), (3, 8, "f64", 700), (4, 3, "f64", 900), (6, 6, "f64", 6),
    (6, 4, "f32", 300), (2, 7, "f64", 500),
])
def test_autotune_then_parity(gpu_lib, d, n, prec, batch):
    variant, param, us = kb.autotune(d, n, prec, batch=batch)
    assert variant in kb.VARIANTS.values() and us > 0
    assert kb.tune_get(d, n, prec) == (variant, param)
    _batched(d, n, batch, prec, 40 + d * 10 + n)


@pytest.mark.parametrize("d,n,prec,batch,variant,param", [
    (6, 4, "f64", 70, "pipe", 0), (6, 4, "f64", 70, "sq", 1), (6, 4, "f64", 70, "sq", 2),
    (6, 4, "f64", 70, "gen", 0), (6, 4, "f64", 70, "large", 0),
    (3, 8, "f64", 90, "mma8", 0), (3, 8, "f64", 90, "sq", 4), (3, 8, "f64", 90, "gen", 0),
    (5, 3, "f64", 90, "sq", 3), (5, 3, "f64", 90, "pipe", 0),
    (6, 6, "f64", 5, "big", 1), (6, 6, "f64", 5, "big", 2), (6, 6, "f64", 5, "big", 4),
    (6, 6, "f64", 5, "big", kb.BIG_SMEM_W),
    (6, 6, "f64", 5, "large", 0),
    (6, 8, "f64", 3, "big", 2), (6, 8, "f64", 3, "big", 2 | kb.BIG_CUDA_CORES),
    (6, 8, "f64", 3, "big", 1 | kb.BIG_CUDA_CORES),
    (6, 4, "f32", 70, "sq", 2), (6, 4, "f32", 70, "gen", 0),
    # a variant that cannot run the shape falls back to the built-in choice
    (4, 3, "f64", 50, "mma8", 0), (6, 6, "f64", 3, "pipe", 0),
])
def test_forced_variant_parity(gpu_lib, d, n, prec, batch, variant, param):
    kb.tune_set(d, n, prec, variant, param)
    _batched(d, n, batch, prec, 70 + d * 10 + n + param, with_w=(variant == "large"))


def test_forced_sq_with_aliasing_outputs(gpu_lib):
    """pbatched with outputs aliased in pairs under a forced entries-per-block
    choice (atomic accumulation with run merging)."""
    d, n, batch = 4, 4, 61
    rng = np.random.default_rng(5)
    L = n ** d
    A = rng.uniform(-1, 1, n * n * d * batch)
    X = rng.uniform(-1, 1, L * batch)
    ny = (batch + 1) // 2
    Y0 = rng.uniform(-1, 1, L * ny)
    Yref = Y0.copy()
    ap = [A.ctypes.data + 8 * (k * d + l) * n * n for k in range(batch) for l in range(d)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * L * (k // 2) for k in range(batch)]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
    for ng in (1, 2, 5):
        kb.tune_set(d, n, "f64", "sq", ng)
        dA, dX, dY = dev(A), dev(X), dev(Y0)
        pX = ptrs(dX, [L * k for k in range(batch)])
        pY = ptrs(dY, [L * (k // 2) for k in range(batch)])
        kb.kronmult_pbatched(d, n, dA, pX, pY)
        assert rel_err(host(dY), Yref) <= TOL["f64"]
