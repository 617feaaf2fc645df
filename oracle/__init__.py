"""ORACLE -- test infrastructure only.

ctypes wrappers over
  * ``oracle/liboracle.so``  -- the plain-C restatement (kron_oracle.c), and
  * ``oracle/_ref/libkronref_{recur,alg993}.so`` -- the reference KRONMULT CPU
    (OpenMP) implementation compiled from its own headers (ref_shim.cpp).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, and only as the checker / the timed CPU baseline.
The product library (``kronmult_b200``) never imports it.

All arrays are numpy float64 in the reference's column-major conventions:
A_l(i, j) at ``A[i + j*ld]``; kron(A_1..A_d) has A_d's index fastest.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def build(with_reference: bool | None = None) -> None:
    """Compile liboracle.so (and the reference CPU build when its sources exist)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    ref_dir = os.environ.get("KRON_REFERENCE_DIR", "/root/reference")
    if with_reference is None:
        with_reference = os.path.isdir(ref_dir)
    if with_reference:
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={ref_dir}"], check=True)


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build(with_reference=False)
        lib = C.CDLL(path)
        lib.oracle_kron_apply.argtypes = [C.c_int, _ip, _ip, _vp, _ip, _dp, _dp, _dp]
        lib.oracle_kron_dense.argtypes = [C.c_int, _ip, _ip, _vp, _ip, _dp, _dp]
        lib.oracle_work_size.argtypes = [C.c_int, _ip, _ip]
        lib.oracle_work_size.restype = C.c_long
        lib.oracle_kronmult_batched.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
        lib.oracle_kronmult_general.argtypes = [C.c_int, _ip, _ip, _vp, _ip, _vp, _vp, C.c_int]
        lib.oracle_kgemm_batched.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                             _vp, _ip, _vp, _ip, C.c_double, _vp, _ip, C.c_int]
        for f in ("oracle_kron_flops", "oracle_flops_forward", "oracle_flops_backward"):
            getattr(lib, f).argtypes = [C.c_int, _ip, _ip]
            getattr(lib, f).restype = C.c_double
        lib.oracle_use_forward.argtypes = [C.c_int, _ip, _ip]
        lib.oracle_use_forward.restype = C.c_int
        lib.oracle_num_threads.restype = C.c_int
        lib.oracle_set_threads.argtypes = [C.c_int]
        _LIB = lib
    return _LIB


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _d(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _ptrs(addrs):
    a = np.ascontiguousarray(np.asarray(addrs, dtype=np.uint64))
    return a, a.ctypes.data_as(_vp)


def num_threads() -> int:
    return _lib().oracle_num_threads()


def set_threads(n: int) -> None:
    _lib().oracle_set_threads(int(n))


# ---------------------------------------------------------------- single entry
def kron_apply(mats, x, y, dense: bool = False):
    """y += kron(mats[0], ..., mats[-1]) @ x  (mats: list of 2-D column-major
    arrays given as numpy arrays in Fortran layout or (m, n) arrays)."""
    d = len(mats)
    Fs = [np.asfortranarray(a, dtype=np.float64) for a in mats]
    m, mp = _i([a.shape[0] for a in Fs])
    n, np_ = _i([a.shape[1] for a in Fs])
    ld, ldp = _i([max(1, a.shape[0]) for a in Fs])
    pa, pap = _ptrs([a.ctypes.data for a in Fs])
    x = np.ascontiguousarray(x, dtype=np.float64)
    assert y.dtype == np.float64 and y.flags.c_contiguous
    if dense:
        _lib().oracle_kron_dense(d, mp, np_, pap, ldp, _d(x), _d(y))
    else:
        ws = _lib().oracle_work_size(d, mp, np_)
        work = np.empty(ws, dtype=np.float64)
        _lib().oracle_kron_apply(d, mp, np_, pap, ldp, _d(x), _d(y), _d(work))
    return y


# ---------------------------------------------------------------- batch forms
def kronmult_batched(d, n, A, X, Y):
    """Y(:,k) += kron(A(:,:,1,k)..A(:,:,d,k)) X(:,k).  A flat (n*n*d*batch),
    X/Y flat (n^d * batch).  X is preserved."""
    batch = Y.size // (n ** d) if n > 0 else 0
    _lib().oracle_kronmult_batched(d, n, _d(A), _d(np.ascontiguousarray(X)), _d(Y), batch)
    return Y


def kronmult_general(d, m, n, a_ptrs, ld, x_ptrs, y_ptrs):
    """Pointer-array form (host addresses).  a_ptrs has d*batch entries
    (entry k's A_l at a_ptrs[l + k*d]); outputs may alias."""
    batch = len(x_ptrs)
    m_, mp = _i(m)
    n_, np_ = _i(n)
    ld_, ldp = _i(ld)
    pa, pap = _ptrs(a_ptrs)
    px, pxp = _ptrs(x_ptrs)
    py, pyp = _ptrs(y_ptrs)
    _lib().oracle_kronmult_general(d, mp, np_, pap, ldp, pxp, pyp, batch)


def kgemm_batched(op, mm, nn, kk, alpha, a_ptrs, ldA, b_ptrs, ldB, beta, c_ptrs, ldC):
    """op: 'nn' | 'nt' | 'tt'.  Pointer arrays hold host addresses."""
    opi = {"nn": 0, "nt": 1, "tt": 2}[op]
    batch = len(c_ptrs)
    pa, pap = _ptrs(a_ptrs)
    pb, pbp = _ptrs(b_ptrs)
    pc, pcp = _ptrs(c_ptrs)
    la, lap = _i(ldA)
    lb, lbp = _i(ldB)
    lc, lcp = _i(ldC)
    _lib().oracle_kgemm_batched(opi, mm, nn, kk, float(alpha), pap, lap, pbp, lbp,
                                float(beta), pcp, lcp, batch)


def kron_flops(m, n) -> float:
    m_, mp = _i(m)
    n_, np_ = _i(n)
    return _lib().oracle_kron_flops(len(m), mp, np_)


def flops_forward(m, n) -> float:
    m_, mp = _i(m)
    n_, np_ = _i(n)
    return _lib().oracle_flops_forward(len(m), mp, np_)


def flops_backward(m, n) -> float:
    m_, mp = _i(m)
    n_, np_ = _i(n)
    return _lib().oracle_flops_backward(len(m), mp, np_)


def use_forward(m, n) -> bool:
    m_, mp = _i(m)
    n_, np_ = _i(n)
    return bool(_lib().oracle_use_forward(len(m), mp, np_))


# ------------------------------------------------ reference CPU build (oracle/_ref)
class Reference:
    """The reference's own CPU/OpenMP implementation (variant 'recur' or 'alg993')."""

    def __init__(self, variant: str = "recur"):
        path = os.path.join(_HERE, "_ref", f"libkronref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        lib.ref_kronmult_batched.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int]
        lib.ref_kronmult_pbatched.argtypes = [C.c_int, C.c_int, _dp, _vp, _vp, _vp, C.c_int]
        lib.ref_kronmult_xbatched.argtypes = [C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, _vp,
                                              C.c_int, C.c_int]
        lib.ref_kronmult_vbatched.argtypes = [C.c_int, _ip, _ip, _vp, _vp, _vp, _dp, C.c_size_t,
                                              C.c_int]
        lib.ref_kgemm_batched.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _vp,
                                          _ip, _vp, _ip, C.c_double, _vp, _ip, C.c_int]
        lib.ref_kronmult_vbatched_entries.argtypes = [C.c_int, _ip, _vp, _vp, _vp, C.c_size_t]
        lib.ref_kron_flops.argtypes = [C.c_int, _ip, _ip]
        lib.ref_kron_flops.restype = C.c_double
        lib.ref_uses_alg993.restype = C.c_int
        lib.ref_max_threads.restype = C.c_int
        lib.ref_set_threads.argtypes = [C.c_int]
        self.lib = lib
        self.variant = variant
        assert bool(lib.ref_uses_alg993()) == (variant == "alg993")

    @staticmethod
    def available(variant: str = "recur") -> bool:
        return os.path.exists(os.path.join(_HERE, "_ref", f"libkronref_{variant}.so"))

    def max_threads(self) -> int:
        return self.lib.ref_max_threads()

    def set_threads(self, n: int) -> None:
        self.lib.ref_set_threads(int(n))

    def kronmult_batched(self, d, n, A, X, Y, W=None):
        """Reference kronmult{d}_batched: X and W are clobbered (pass copies)."""
        batch = Y.size // (n ** d)
        if W is None:
            W = np.zeros_like(Y)
        rc = self.lib.ref_kronmult_batched(d, n, _d(A), _d(X), _d(Y), _d(W), batch)
        assert rc == 0

    def kronmult_pbatched(self, d, n, A, x_ptrs, y_ptrs, w_ptrs):
        px, pxp = _ptrs(x_ptrs)
        py, pyp = _ptrs(y_ptrs)
        pw, pwp = _ptrs(w_ptrs)
        rc = self.lib.ref_kronmult_pbatched(d, n, _d(A), pxp, pyp, pwp, len(x_ptrs))
        assert rc == 0

    def kronmult_xbatched(self, d, n, a_ptrs, lda, x_ptrs, y_ptrs, w_ptrs, subbatch=0):
        pa, pap = _ptrs(a_ptrs)
        px, pxp = _ptrs(x_ptrs)
        py, pyp = _ptrs(y_ptrs)
        pw, pwp = _ptrs(w_ptrs)
        rc = self.lib.ref_kronmult_xbatched(d, n, pap, lda, pxp, pyp, pwp, len(x_ptrs), subbatch)
        assert rc == 0

    def kronmult_vbatched(self, d, m, n, a_ptrs, x_ptrs, y_ptrs, W):
        m_, mp = _i(m)
        n_, np_ = _i(n)
        pa, pap = _ptrs(a_ptrs)
        px, pxp = _ptrs(x_ptrs)
        py, pyp = _ptrs(y_ptrs)
        rc = self.lib.ref_kronmult_vbatched(d, mp, np_, pap, pxp, pyp, _d(W), W.nbytes,
                                            len(x_ptrs))
        assert rc == 0

    def kronmult_vbatched_entries(self, shapes, a_ptrs, x_ptrs, y_ptrs, wbytes=1 << 24):
        sh, shp = _i(np.asarray(shapes).reshape(-1))
        pa, pap = _ptrs(a_ptrs)
        px, pxp = _ptrs(x_ptrs)
        py, pyp = _ptrs(y_ptrs)
        rc = self.lib.ref_kronmult_vbatched_entries(len(x_ptrs), shp, pap, pxp, pyp, wbytes)
        assert rc == 0

    def kgemm_batched(self, op, mm, nn, kk, alpha, a_ptrs, ldA, b_ptrs, ldB, beta, c_ptrs, ldC):
        opi = {"nn": 0, "nt": 1, "tt": 2}[op]
        pa, pap = _ptrs(a_ptrs)
        pb, pbp = _ptrs(b_ptrs)
        pc, pcp = _ptrs(c_ptrs)
        la, lap = _i(ldA)
        lb, lbp = _i(ldB)
        lc, lcp = _i(ldC)
        rc = self.lib.ref_kgemm_batched(opi, mm, nn, kk, float(alpha), pap, lap, pbp, lbp,
                                        float(beta), pcp, lcp, len(c_ptrs))
        assert rc == 0

    def kron_flops(self, m, n) -> float:
        m_, mp = _i(m)
        n_, np_ = _i(n)
        return self.lib.ref_kron_flops(len(m), mp, np_)
