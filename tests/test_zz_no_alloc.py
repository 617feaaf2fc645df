"""kronmult_batched_noalloc_async: the batched product for callers that
cannot allocate device memory where they apply the operator (inside a
global-mode stream capture, under a pool that owns all of HBM, or in a
callback that only holds A, X and Y).  It takes no workspace and uses the
library's 16 MiB file-scope device scratch array for vectors that exceed
shared memory.

Checked here through the C ABI against the workspace-taking entry point
kronmult{d}_batched_async, at the FP64 tolerance of the other tests, on two
calls in a row (the array keeps the previous call's contents).  Collected
last so a stopping run has run everything else first."""
import ctypes as C

import numpy as np
import pytest

import kronmult_b200 as kb
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
KRON_ERROR_WORKSPACE = 2


@pytest.mark.parametrize("d,n,batch", [
    (6, 6, 50),   # 373 KB vectors: two-phase path through the scratch, 2 chunks
    (5, 8, 9),    # 262 KB vectors: two-phase path, 1 chunk
    (6, 4, 8),    # fits on chip: no scratch use
])
def test_noalloc_matches_workspace_entry_point(gpu_lib, d, n, batch):
    import torch

    lib = kb.lib()
    rng = np.random.default_rng(4242 + 10 * d + n)
    L = n ** d
    A = dev(rng.standard_normal(n * n * d * batch) / np.sqrt(n))
    X = dev(rng.uniform(-1, 1, L * batch))
    Y0 = rng.uniform(-1, 1, L * batch)
    stream = torch.cuda.current_stream().cuda_stream

    # existing entry point, caller-provided workspace
    need = lib.kron_batched_workspace_bytes(d, n, batch)
    W = torch.empty(max(1, need // 8), dtype=torch.float64, device="cuda") if need else None
    Yref = dev(Y0)
    f = getattr(lib, f"kronmult{d}_batched_async")
    assert f(n, A.data_ptr(), X.data_ptr(), Yref.data_ptr(),
             None if W is None else W.data_ptr(), batch, stream) == 0
    ref = host(Yref)

    # the no-allocation entry point, twice in a row
    for _ in range(2):
        Yn = dev(Y0)
        rc = lib.kronmult_batched_noalloc_async(d, n, A.data_ptr(), X.data_ptr(), Yn.data_ptr(),
                                                batch, stream)
        assert rc == 0
        assert rel_err(host(Yn), ref) <= TOL64


def test_noalloc_rejects_vectors_beyond_the_scratch(gpu_lib):
    # 12^6 doubles exceed the 16 MiB array: refused before anything is touched
    rc = kb.lib().kronmult_batched_noalloc_async(6, 12, None, None, None, 1, None)
    assert rc == KRON_ERROR_WORKSPACE
