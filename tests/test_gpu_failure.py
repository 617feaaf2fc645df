"""GPU: the library's failure paths, driven from the host.  No test here
faults, traps or hangs a GPU.

- Wait time-out: a bound of one poll (kron_set_wait_limit) makes the
  pipelined kernel (d = 6, n = 4) and the slab-cluster kernel (d = 6, n = 6)
  give up on their first asynchronous copy, and the tensor-core split
  kernels (d = 6, n = 8) on their first MMA commit.  The copies still land (the
  drain keeps the full bound) and the kernels return.  The status word then
  reads 1, and the next call with the default bound is clean and correct.
- Allocation failure: an injected device-allocation failure
  (kron_test_fail_alloc) makes kron_segments_create, kron_vplan_create and
  kron_autotune return KRON_ERROR_ALLOC with nothing left allocated
  (kron_test_live_allocs) and no plan returned.

The reference checks its HIP calls with assert(istat == hipSuccess) only
(test_kronmult6_batched.cpp:215-216); these paths have no counterpart
there."""
import ctypes as C

import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

ALLOC = 5  # KRON_ERROR_ALLOC


@pytest.fixture(autouse=True)
def _restore():
    kb.tune_clear()
    yield
    kb.lib().kron_set_wait_limit(0)
    kb.lib().kron_test_fail_alloc(-1)
    kb.tune_clear()


@pytest.mark.parametrize("n,variant,batch", [(4, "pipe", 2000), (6, "slab", 90)])
def test_wait_timeout_then_clean(gpu_lib, n, variant, batch):
    import torch

    lib = kb.lib()
    d, L = 6, n ** 6
    rng = np.random.default_rng(700 + n)
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * batch)
    kb.tune_set(d, n, "f64", variant, 0)
    dA, dX = dev(A), dev(X)
    assert lib.kron_device_status(1) in (0, 1)
    assert lib.kron_set_wait_limit(1) == 0
    dY = dev(Y0)
    kb.kronmult_batched(d, n, dA, dX, dY, None)
    torch.cuda.synchronize()
    assert lib.kron_set_wait_limit(0) == 0
    assert lib.kron_device_status(1) == 1, "the one-poll wait should have run out"
    assert lib.kron_device_status(0) == 0, "the status word was cleared"
    # the context is usable and the default bound gives the right answer
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    dY = dev(Y0)
    kb.kronmult_batched(d, n, dA, dX, dY, None)
    assert rel_err(host(dY), Yref) <= 1e-13
    assert lib.kron_device_status(1) == 0


def test_wait_timeout_tensor_core_split_then_clean(gpu_lib):
    """The tcgen05 split kernels (d = 6, n = 8): with a one-poll bound the
    wait for the first commit of the MMAs runs out; each block waits for its
    MMAs with the full drain bound, frees its tensor memory and leaves."""
    import torch

    lib = kb.lib()
    d, n, batch = 6, 8, 2
    L = n ** d
    rng = np.random.default_rng(708)
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * batch)
    kb.tune_set(d, n, "split", "split_tc")
    dA, dX = dev(A), dev(X)
    W = torch.empty(L * batch, dtype=torch.float64, device="cuda")
    assert lib.kron_device_status(1) in (0, 1)
    assert lib.kron_set_wait_limit(1) == 0
    kb.kronmult_batched_split(d, n, dA, dX, dev(Y0), W)
    torch.cuda.synchronize()
    assert lib.kron_set_wait_limit(0) == 0
    assert lib.kron_device_status(1) == 1, "the one-poll wait should have run out"
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    dY = dev(Y0)
    kb.kronmult_batched_split(d, n, dA, dX, dY, W)
    assert rel_err(host(dY), Yref) <= 1e-12
    assert lib.kron_device_status(1) == 0


def test_set_wait_limit_rejects_negative(gpu_lib):
    assert kb.lib().kron_set_wait_limit(-5) == 1


def _segments_create(lib, pY, batch):
    plan = C.c_void_p()
    rc = lib.kron_segments_create(C.byref(plan), pY.data_ptr(), batch, None)
    return rc, plan


def test_alloc_failure_segments(gpu_lib):
    lib = kb.lib()
    import torch

    batch, L = 50, 64
    Y = torch.zeros(L * 20, dtype=torch.float64, device="cuda")
    pY = ptrs(Y, [L * (k % 20) for k in range(batch)])
    base = lib.kron_test_live_allocs()
    for nth in (0, 1):  # the plan makes two device allocations
        assert lib.kron_test_fail_alloc(nth) == 0
        rc, plan = _segments_create(lib, pY, batch)
        assert rc == ALLOC and not plan.value
        assert lib.kron_test_live_allocs() == base
    rc, plan = _segments_create(lib, pY, batch)
    assert rc == 0 and plan.value
    assert lib.kron_segments_count(plan) == 20
    assert lib.kron_test_live_allocs() == base + 2
    assert lib.kron_segments_destroy(plan) == 0
    assert lib.kron_test_live_allocs() == base


def test_alloc_failure_vplan(gpu_lib):
    lib = kb.lib()
    rng = np.random.default_rng(710)
    nent = 40
    shapes = np.zeros((nent, 13), dtype=np.int32)
    for k in range(nent):
        d = int(rng.integers(1, 7))
        shapes[k, 0] = d
        shapes[k, 1:1 + 2 * d] = rng.choice([2, 3, 4, 6, 8], size=2 * d)
    shapes[0, 0], shapes[0, 1:13] = 6, 8  # one entry beyond shared memory: work items
    base = lib.kron_test_live_allocs()
    for nth in (0, 1, 2):  # counters, entry descriptors, work items
        assert lib.kron_test_fail_alloc(nth) == 0
        plan = C.c_void_p()
        rc = lib.kron_vplan_create(C.byref(plan), nent, shapes.ctypes.data)
        assert rc == ALLOC and not plan.value
        assert lib.kron_test_live_allocs() == base
    plan = C.c_void_p()
    assert lib.kron_vplan_create(C.byref(plan), nent, shapes.ctypes.data) == 0
    assert lib.kron_test_live_allocs() > base
    assert lib.kron_vplan_destroy(plan) == 0
    assert lib.kron_test_live_allocs() == base


def test_alloc_failure_autotune(gpu_lib):
    lib = kb.lib()
    base = lib.kron_test_live_allocs()
    for nth in (0, 1, 2, 3):  # A, X, Y, W of the synthetic problem
        assert lib.kron_test_fail_alloc(nth) == 0
        v, q, t = C.c_int(-1), C.c_int(-1), C.c_double(-1.0)
        rc = lib.kron_autotune(6, 4, 0, 64, C.byref(v), C.byref(q), C.byref(t), None)
        assert rc == ALLOC
        assert v.value == -1, "no choice is reported on failure"
        assert kb.tune_get(6, 4, "f64") == (None, 0), "nothing is recorded on failure"
        assert lib.kron_test_live_allocs() == base
    lib.kron_test_fail_alloc(-1)
    variant, _, us = kb.autotune(6, 4, "f64", batch=64)
    assert variant in kb.VARIANTS.values() and us > 0
    assert lib.kron_test_live_allocs() == base


def test_alloc_failure_fp64_probe(gpu_lib):
    lib = kb.lib()
    base = lib.kron_test_live_allocs()
    lib.kron_test_fail_alloc(0)
    t, c = C.c_double(), C.c_double()
    assert lib.kron_measure_fp64_peak(C.byref(t), C.byref(c)) == ALLOC
    assert lib.kron_test_live_allocs() == base
