"""CPU-side checks of the C ABI: the library loads, exports every symbol
include/kronmult.h declares (C++-linkage reference names included), and the
host-side argument validation answers without touching a GPU."""
import ctypes as C
import re
import subprocess

import pytest

import kronmult_b200 as kb


@pytest.fixture(scope="module")
def lib():
    return kb.lib()


def _exported():
    out = subprocess.run(["nm", "-DC", "--defined-only", kb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return out


def test_library_loads(lib):
    assert lib.kron_version().decode().count(".") == 2
    assert lib.kron_status_string(0) == b"KRON_SUCCESS"


def test_every_declared_symbol_is_exported(lib):
    exported = _exported()
    names = kb.declared_symbols()
    assert len(names) >= 70
    for name in names:
        if hasattr(lib, name):
            continue
        # C++ linkage: demangled "name(" must be present
        assert re.search(r"\b" + re.escape(name) + r"\(", exported), name


def test_reference_mangled_names():
    out = subprocess.run(["nm", "-D", "--defined-only", kb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    # the reference wrappers' symbols (kronmult6_batched.cpp:4-5,
    # kronmult6_xbatched.cpp:4-7, kgemm_nt_batched.cpp:5-10)
    for sym in ("_Z17kronmult6_batchediPKdPdS1_S1_i",
                "_Z18kronmult6_xbatchediPKPKdiPPdS4_S4_ii",
                "_Z18kronmult6_pbatchediPKdPPdS2_S2_i",
                "_Z16kgemm_nt_batchediiidPKPdPKiS1_S3_dS1_S3_i"):
        assert sym in out, sym


def test_validation_without_gpu(lib):
    # d out of range / negative sizes -> INVALID_VALUE, before any launch
    assert lib.kronmult_batched_f32_async(7, 4, None, None, None, None, 1, None) == 1
    assert lib.kronmult6_batched_async(-1, None, None, None, None, 1, None) == 1
    assert lib.kronmult6_batched_async(4, None, None, None, None, -3, None) == 1
    # empty batch is a successful no-op
    assert lib.kronmult6_batched_async(4, None, None, None, None, 0, None) == 0
    # null operands with work to do
    assert lib.kronmult3_pbatched_async(4, None, None, None, None, 5, None) == 1
    # xbatched: lda < n
    assert lib.kronmult3_xbatched_async(4, C.c_void_p(8), 3, C.c_void_p(8), C.c_void_p(8),
                                        None, 2, 0, None) == 1
    assert lib.kgemm_nn_batched_async(-1, 2, 2, 1.0, None, None, None, None, 0.0, None, None, 1,
                                      None) == 1
    assert lib.kgemm_tt_batched_async(2, 2, 2, 1.0, None, None, None, None, 0.0, None, None, 0,
                                      None) == 0


def test_last_status_of_reference_signatures(lib):
    lib.kron_clear_last_status()
    assert lib.kron_get_last_status() == 0


def test_kron_flops_c_matches_oracle():
    import numpy as np

    import oracle

    rng = np.random.default_rng(5)
    for _ in range(50):
        d = int(rng.integers(1, 7))
        m = rng.integers(1, 9, size=d).astype(np.int32)
        n = rng.integers(1, 9, size=d).astype(np.int32)
        got = kb.lib().kron_flops_c(d, m.ctypes.data, n.ctypes.data)
        assert got == oracle.kron_flops(m, n)


def test_vplan_rejects_bad_shapes(lib):
    import numpy as np

    h = C.c_void_p()
    bad = np.zeros((1, 13), dtype=np.int32)
    bad[0, 0] = 7
    assert lib.kron_vplan_create(C.byref(h), 1, bad.ctypes.data) == 1
    bad[0, 0] = 2
    bad[0, 1:5] = [2, 0, 3, 3]
    assert lib.kron_vplan_create(C.byref(h), 1, bad.ctypes.data) == 1
