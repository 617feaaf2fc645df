"""kronmult_b200 -- batched Kronecker matrix-vector products on B200 (sm_100a).

The product is the C-ABI shared library ``kronmult_b200/lib/libkronmult_b200.so``
(declared in ``include/kronmult.h``).  This module loads it with ctypes and
offers thin wrappers that take torch CUDA tensors (device memory and streams
come from PyTorch; all arithmetic runs in the library's CUDA kernels).  There
is no CPU fallback: if the library is missing or no GPU is present, calls
raise.

Layouts follow the reference KRONMULT (column major, A_d's index fastest):
  batched   A (n,n,d,batch) flat, X/Y (n^d, batch) flat
  pbatched  A as batched, X/Y as tensors of device pointers (int64)
  xbatched  A as a tensor of d*batch device pointers, common lda
  vbatched  rectangular shapes, A pointers with ld = m_l
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libkronmult_b200.so")
INCLUDE_H = os.path.join(os.path.dirname(HERE), "include", "kronmult.h")

_LIB = None

KRON_SUCCESS = 0
STATUS = {0: "KRON_SUCCESS", 1: "KRON_ERROR_INVALID_VALUE", 2: "KRON_ERROR_WORKSPACE",
          3: "KRON_ERROR_LAUNCH", 4: "KRON_ERROR_NOT_SUPPORTED", 5: "KRON_ERROR_ALLOC",
          6: "KRON_ERROR_INTERNAL"}


class KronError(RuntimeError):
    def __init__(self, status, what=""):
        super().__init__(f"{what}: {STATUS.get(status, status)}")
        self.status = status


def build(verbose: bool = False) -> str:
    from . import builder as _b

    return _b.build(verbose=verbose)


_i, _d, _vp, _sz = C.c_int, C.c_double, C.c_void_p, C.c_size_t


def _sig(lib):
    S = {}
    for D in range(1, 7):
        S[f"kronmult{D}_batched_async"] = [_i, _vp, _vp, _vp, _vp, _i, _vp]
        S[f"kronmult{D}_pbatched_async"] = [_i, _vp, _vp, _vp, _vp, _i, _vp]
        S[f"kronmult{D}_xbatched_async"] = [_i, _vp, _i, _vp, _vp, _vp, _i, _i, _vp]
        S[f"kronmult{D}_vbatched_async"] = [_i] * (2 * D) + [_vp, _vp, _vp, _vp, _sz, _i, _vp]
    for op in ("nn", "nt", "tt"):
        S[f"kgemm_{op}_batched_async"] = [_i, _i, _i, _d, _vp, _vp, _vp, _vp, _d, _vp, _vp, _i,
                                          _vp]
    S["kron_batched_workspace_bytes"] = [_i, _i, _i]
    S["kron_vbatched_workspace_bytes"] = [_i, _vp, _vp, _i]
    S["kronmult_batched_f32_async"] = [_i, _i, _vp, _vp, _vp, _vp, _i, _vp]
    S["kronmult_batched_split_async"] = [_i, _i, _vp, _vp, _vp, _vp, _i, _vp]
    S["kronmult_batched_noalloc_async"] = [_i, _i, _vp, _vp, _vp, _i, _vp]
    S["kron_segments_create"] = [_vp, _vp, _i, _vp]
    S["kron_segments_destroy"] = [_vp]
    S["kron_segments_count"] = [_vp]
    S["kronmult_xbatched_segmented_async"] = [_i, _i, _vp, _i, _vp, _vp, _vp, _i, _vp, _vp]
    S["kronmult_pbatched_segmented_async"] = [_i, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp]
    S["kron_vplan_create"] = [_vp, _i, _vp]
    S["kron_vplan_destroy"] = [_vp]
    S["kron_vplan_workspace_bytes"] = [_vp]
    S["kron_vplan_flops"] = [_vp]
    S["kron_vplan_execute_async"] = [_vp, _vp, _vp, _vp, _vp, _sz, _vp]
    S["kron_flops_c"] = [_i, _vp, _vp]
    S["kron_status_string"] = [_i]
    S["kron_get_last_status"] = []
    S["kron_clear_last_status"] = []
    S["kron_version"] = []
    S["kron_measure_fp64_peak"] = [_vp, _vp]
    S["kron_device_status"] = [_i]
    S["kron_set_wait_limit"] = [C.c_longlong]
    S["kron_test_fail_alloc"] = [_i]
    S["kron_test_live_allocs"] = []
    S["kron_build_pointers_async"] = [_i, _i, _vp, C.c_longlong, _vp, _vp, C.c_longlong, _vp,
                                      _vp, C.c_longlong, _vp, _vp, _vp, _vp, _vp]
    S["kron_owner_partition"] = [_i, _vp, _i, _vp, _vp, _vp]
    S["kron_l2_persist_async"] = [_vp, _sz, _vp]
    S["kron_l2_persist_reset"] = [_vp]
    S["kron_autotune"] = [_i, _i, _i, _i, _vp, _vp, _vp, _vp]
    S["kron_tune_set"] = [_i, _i, _i, _i, _i]
    S["kron_tune_get"] = [_i, _i, _i, _vp, _vp]
    S["kron_tune_clear"] = []
    S["kron_tune_save"] = [C.c_char_p]
    S["kron_tune_load"] = [C.c_char_p]
    for name, args in S.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = _i
    lib.kron_batched_workspace_bytes.restype = _sz
    lib.kron_vbatched_workspace_bytes.restype = _sz
    lib.kron_vplan_workspace_bytes.restype = _sz
    lib.kron_vplan_flops.restype = _d
    lib.kron_flops_c.restype = _d
    lib.kron_status_string.restype = C.c_char_p
    lib.kron_version.restype = C.c_char_p
    lib.kron_tune_clear.restype = None
    lib.kron_test_live_allocs.restype = C.c_longlong
    return lib


def lib():
    """Load libkronmult_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `python -m kronmult_b200.builder`")
        _LIB = _sig(C.CDLL(LIB_PATH))
    return _LIB


def declared_symbols():
    """Function names declared in include/kronmult.h (extern "C" and C++)."""
    import re

    txt = open(INCLUDE_H).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:int|void|size_t|double|char)\s*\*?\s*(\w+)\s*\(",
                       txt, flags=re.M)
    return sorted(set(names))


# ---------------------------------------------------------------- torch helpers
def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("kronmult_b200 needs a CUDA device")
    return torch


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream(stream):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _check(rc, what):
    if rc != KRON_SUCCESS:
        raise KronError(rc, what)


def kronmult_batched(d, n, A, X, Y, W=None, stream=None):
    """Y(:,k) += kron(A_1..A_d)(k) X(:,k) -- kronmult{d}_batched."""
    f = getattr(lib(), f"kronmult{d}_batched_async")
    batch = Y.numel() // (n ** d) if n else 0
    _check(f(n, _ptr(A), _ptr(X), _ptr(Y), _ptr(W), batch, _stream(stream)),
           f"kronmult{d}_batched")


def kronmult_pbatched(d, n, A, pX, pY, pW=None, stream=None):
    f = getattr(lib(), f"kronmult{d}_pbatched_async")
    _check(f(n, _ptr(A), _ptr(pX), _ptr(pY), _ptr(pW), pX.numel(), _stream(stream)),
           f"kronmult{d}_pbatched")


def kronmult_xbatched(d, n, pA, lda, pX, pY, pW=None, subbatch=0, stream=None):
    f = getattr(lib(), f"kronmult{d}_xbatched_async")
    _check(f(n, _ptr(pA), lda, _ptr(pX), _ptr(pY), _ptr(pW), pX.numel(), subbatch,
             _stream(stream)), f"kronmult{d}_xbatched")


def kronmult_vbatched(m, n, pA, pX, pY, W=None, stream=None):
    d = len(m)
    f = getattr(lib(), f"kronmult{d}_vbatched_async")
    mn = []
    for a, b in zip(m, n):
        mn += [a, b]
    wbytes = 0 if W is None else W.numel() * W.element_size()
    _check(f(*mn, _ptr(pA), _ptr(pX), _ptr(pY), _ptr(W), wbytes, pX.numel(), _stream(stream)),
           f"kronmult{d}_vbatched")


def kgemm_batched(op, mm, nn, kk, alpha, pA, ldA, pB, ldB, beta, pC, ldC, stream=None):
    f = getattr(lib(), f"kgemm_{op}_batched_async")
    _check(f(mm, nn, kk, float(alpha), _ptr(pA), _ptr(ldA), _ptr(pB), _ptr(ldB), float(beta),
             _ptr(pC), _ptr(ldC), pC.numel(), _stream(stream)), f"kgemm_{op}_batched")


def kronmult_batched_f32(d, n, A, X, Y, W=None, stream=None):
    batch = Y.numel() // (n ** d)
    _check(lib().kronmult_batched_f32_async(d, n, _ptr(A), _ptr(X), _ptr(Y), _ptr(W), batch,
                                            _stream(stream)), "kronmult_batched_f32")


def kronmult_batched_split(d, n, A, X, Y, W=None, stream=None):
    batch = Y.numel() // (n ** d)
    _check(lib().kronmult_batched_split_async(d, n, _ptr(A), _ptr(X), _ptr(Y), _ptr(W), batch,
                                              _stream(stream)), "kronmult_batched_split")


def measure_fp64_peak():
    """(tensor, cuda_core) FP64 TFLOP/s of the current device."""
    a, b = C.c_double(), C.c_double()
    _check(lib().kron_measure_fp64_peak(C.byref(a), C.byref(b)), "kron_measure_fp64_peak")
    return a.value, b.value


def build_pointers(d, A, astride, alist, X, xstride, xlist, Y, ystride, ylist, stream=None):
    """Device pointer arrays (pA, pX, pY) of the xbatched / pbatched layouts
    from device int32 index lists (None: identity):
    pX[k] = X + xlist[k]*xstride, pY[k] = Y + ylist[k]*ystride,
    pA[l + k*d] = A + alist[l + k*d]*astride (strides in elements)."""
    torch = _torch()
    batch = next(v.numel() for v in (xlist, ylist) if v is not None) if (
        xlist is not None or ylist is not None) else alist.numel() // d
    pA = torch.empty(batch * d, dtype=torch.int64, device="cuda")
    pX = torch.empty(batch, dtype=torch.int64, device="cuda")
    pY = torch.empty(batch, dtype=torch.int64, device="cuda")
    _check(lib().kron_build_pointers_async(d, batch, _ptr(A), astride, _ptr(alist), _ptr(X),
                                           xstride, _ptr(xlist), _ptr(Y), ystride, _ptr(ylist),
                                           _ptr(pA), _ptr(pX), _ptr(pY), _stream(stream)),
           "kron_build_pointers")
    return pA, pX, pY


def l2_persist(t, stream=None):
    """Keep tensor t (e.g. the factors A of a repeated apply) resident in L2
    for the library's kernels on `stream`."""
    _check(lib().kron_l2_persist_async(_ptr(t), t.numel() * t.element_size(), _stream(stream)),
           "kron_l2_persist")


def l2_persist_reset(stream=None):
    _check(lib().kron_l2_persist_reset(_stream(stream)), "kron_l2_persist_reset")


# ---------------------------------------------------------------- autotuner
PRECISIONS = {"f64": 0, "f32": 1, "split": 2}
VARIANTS = {1: "mma8", 2: "pipe", 3: "sq", 4: "gen", 5: "big", 6: "large", 7: "slab",
            8: "split_tc"}
# "big" param bit: FP64 d = 6, n = 8 on CUDA-core FMAs instead of tensor cores
BIG_CUDA_CORES = 256
# "big" param bit: keep the intermediate in the cluster's shared memory
# instead of the workspace W (FP64 d = 6, n = 6)
BIG_SMEM_W = 512
# "big" param bit: no L2 cache policies on W, x and y (comparison form)
BIG_NO_L2_HINTS = 1024
# "slab" param bit: no lane rotation in the first FP64 pass (comparison form)
SLAB_NO_ROTATE = 1
# "slab" param bit: clusters of 6 blocks holding whole slabs (comparison form)
SLAB_WHOLE = 2
# "slab" param bit: distinct outputs by loads and stores (comparison form)
SLAB_PLAIN_Y = 4
# "slab" param bit: no side kernel on the SMs the slab clusters leave idle
SLAB_NO_SIDE = 8


def autotune(d, n, precision="f64", batch=1024, stream=None):
    """Time every kernel variant for square (d, n) at `precision` on a
    synthetic batch and record the fastest; returns (variant, param, us)."""
    v, q, t = C.c_int(), C.c_int(), C.c_double()
    _check(lib().kron_autotune(d, n, PRECISIONS[precision], batch, C.byref(v), C.byref(q),
                               C.byref(t), _stream(stream)), "kron_autotune")
    return VARIANTS[v.value], q.value, t.value


def tune_set(d, n, precision, variant, param=0):
    """Record a variant by name ("sq", "big", ...; None removes the entry)."""
    code = 0 if variant is None else {v: k for k, v in VARIANTS.items()}[variant]
    _check(lib().kron_tune_set(d, n, PRECISIONS[precision], code, param), "kron_tune_set")


def tune_get(d, n, precision="f64"):
    """(variant name or None, param) recorded for (d, n, precision)."""
    v, q = C.c_int(), C.c_int()
    _check(lib().kron_tune_get(d, n, PRECISIONS[precision], C.byref(v), C.byref(q)),
           "kron_tune_get")
    return VARIANTS.get(v.value), q.value


def tune_clear():
    lib().kron_tune_clear()


def tune_save(path):
    _check(lib().kron_tune_save(os.fsencode(path)), "kron_tune_save")


def tune_load(path):
    _check(lib().kron_tune_load(os.fsencode(path)), "kron_tune_load")


class Segments:
    """Deterministic accumulation plan (groups entries by output pointer)."""

    def __init__(self, pY, stream=None):
        h = C.c_void_p()
        _check(lib().kron_segments_create(C.byref(h), _ptr(pY), pY.numel(), _stream(stream)),
               "kron_segments_create")
        self.handle = h
        self.batch = pY.numel()

    @property
    def count(self):
        return lib().kron_segments_count(self.handle)

    def close(self):
        if self.handle:
            lib().kron_segments_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kronmult_xbatched_segmented(d, n, pA, lda, pX, pY, seg, pW=None, stream=None):
    _check(lib().kronmult_xbatched_segmented_async(d, n, _ptr(pA), lda, _ptr(pX), _ptr(pY),
                                                   _ptr(pW), pX.numel(), seg.handle,
                                                   _stream(stream)),
           "kronmult_xbatched_segmented")


def kronmult_pbatched_segmented(d, n, A, pX, pY, seg, pW=None, stream=None):
    _check(lib().kronmult_pbatched_segmented_async(d, n, _ptr(A), _ptr(pX), _ptr(pY), _ptr(pW),
                                                   pX.numel(), seg.handle, _stream(stream)),
           "kronmult_pbatched_segmented")


class VPlan:
    """Uneven-batch plan; shapes is a host int array of 13 ints per entry."""

    def __init__(self, shapes):
        import numpy as np

        arr = np.ascontiguousarray(np.asarray(shapes, dtype=np.int32).reshape(-1, 13))
        h = C.c_void_p()
        _check(lib().kron_vplan_create(C.byref(h), arr.shape[0], arr.ctypes.data),
               "kron_vplan_create")
        self.handle = h
        self.batch = arr.shape[0]

    @property
    def workspace_bytes(self):
        return lib().kron_vplan_workspace_bytes(self.handle)

    @property
    def flops(self):
        return lib().kron_vplan_flops(self.handle)

    def execute(self, pA, pX, pY, W=None, stream=None):
        wbytes = 0 if W is None else W.numel() * W.element_size()
        _check(lib().kron_vplan_execute_async(self.handle, _ptr(pA), _ptr(pX), _ptr(pY), _ptr(W),
                                              wbytes, _stream(stream)), "kron_vplan_execute")

    def close(self):
        if self.handle:
            lib().kron_vplan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
