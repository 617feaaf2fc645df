"""kron_build_pointers_async argument checks (rejected before any device work)."""
import ctypes as C

import pytest

import kronmult_b200 as kb


@pytest.mark.parametrize("d,batch,astride,xstride,ystride", [
    (0, 4, 1, 1, 1), (7, 4, 1, 1, 1), (3, -1, 1, 1, 1), (3, 4, -1, 1, 1), (3, 4, 1, -2, 1),
    (3, 4, 1, 1, -3),
])
def test_rejects_bad_arguments(d, batch, astride, xstride, ystride):
    rc = kb.lib().kron_build_pointers_async(d, batch, None, astride, None, None, xstride, None,
                                            None, ystride, None, None, None, None, None)
    assert rc == 1  # KRON_ERROR_INVALID_VALUE


def test_output_without_base_is_rejected():
    dummy = C.c_void_p(16)
    rc = kb.lib().kron_build_pointers_async(3, 4, None, 16, None, None, 64, None, None, 64, None,
                                            dummy, None, None, None)
    assert rc == 1


def test_nothing_to_build_is_success():
    assert kb.lib().kron_build_pointers_async(3, 0, None, 1, None, None, 1, None, None, 1, None,
                                              None, None, None, None) == 0


def test_l2_persist_rejects_empty_range():
    assert kb.lib().kron_l2_persist_async(None, 1024, None) == 1
    assert kb.lib().kron_l2_persist_async(C.c_void_p(256), 0, None) == 1
