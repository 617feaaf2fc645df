"""kronmult_batched_noalloc_async: the batched product for callers that
cannot allocate device memory where they apply the operator (inside a
global-mode stream capture, under a pool that owns all of HBM, or in a
callback that only holds A, X and Y).  It takes no workspace and uses the
library's 16 MiB file-scope device scratch array for vectors that exceed
shared memory.

Checked here through the C ABI against the oracle and against the
workspace-taking entry point kronmult{d}_batched_async, at the FP64
tolerance of the other tests, on two calls in a row (the array keeps the
previous call's contents).  Forced kernel variants send d = 6, n = 6 through
each form that uses the array (two-phase launches, the cluster two-phase
kernel) with a batch that spans two chunks of it, and through the forms that
need none (slab-cluster kernel, cluster shared-memory form).  Collected last
so a stopping run has run everything else first."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
KRON_ERROR_WORKSPACE = 2


@pytest.fixture(autouse=True)
def _clean_table():
    kb.tune_clear()
    yield
    kb.tune_clear()


@pytest.mark.parametrize("d,n,batch,variant,param", [
    (6, 6, 50, None, 0),        # built-in choice: slab-cluster kernel, no scratch
    (6, 6, 50, "large", 0),     # two-phase launches through the scratch, 2 chunks (44 + 6)
    (6, 6, 50, "big", 2),       # cluster two-phase kernel through the scratch, 2 chunks
    (6, 6, 50, "big", kb.BIG_SMEM_W),  # intermediate in cluster shared memory
    (5, 8, 9, None, 0),         # 262 KB vectors: cluster two-phase through the scratch
    (6, 4, 8, None, 0),         # fits on chip: no scratch use
])
def test_noalloc_matches_oracle_and_workspace_entry_point(gpu_lib, d, n, batch, variant, param):
    import torch

    lib = kb.lib()
    if variant is not None:
        kb.tune_set(d, n, "f64", variant, param)
    rng = np.random.default_rng(4242 + 10 * d + n + param)
    L = n ** d
    A_h = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X_h = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * batch)
    A, X = dev(A_h), dev(X_h)
    stream = torch.cuda.current_stream().cuda_stream

    expect = Y0.copy()
    oracle.kronmult_batched(d, n, A_h, X_h, expect)

    # existing entry point, caller-provided workspace
    need = max(lib.kron_batched_workspace_bytes(d, n, batch), 8 * L * batch)
    W = torch.empty(max(1, need // 8), dtype=torch.float64, device="cuda")
    Yref = dev(Y0)
    f = getattr(lib, f"kronmult{d}_batched_async")
    assert f(n, A.data_ptr(), X.data_ptr(), Yref.data_ptr(), W.data_ptr(), batch, stream) == 0
    ref = host(Yref)
    assert rel_err(ref, expect) <= TOL64

    # the no-allocation entry point, twice in a row
    for _ in range(2):
        Yn = dev(Y0)
        rc = lib.kronmult_batched_noalloc_async(d, n, A.data_ptr(), X.data_ptr(), Yn.data_ptr(),
                                                batch, stream)
        assert rc == 0
        got = host(Yn)
        assert rel_err(got, expect) <= TOL64
        assert rel_err(got, ref) <= TOL64
    assert lib.kron_device_status(1) == 0


def test_noalloc_rejects_vectors_beyond_the_scratch(gpu_lib):
    # 12^6 doubles exceed the 16 MiB array: refused before anything is touched
    rc = kb.lib().kronmult_batched_noalloc_async(6, 12, None, None, None, 1, None)
    assert rc == KRON_ERROR_WORKSPACE
