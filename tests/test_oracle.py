"""The oracle (plain-C restatement) pinned against the reference's own
outputs (golden vectors) and the reference tests' dense-Kronecker check."""
import numpy as np
import pytest

import oracle
from tests.golden_cases import rel_err

TOL = 1e-13  # FP64, different summation order than the reference


def _square_mats(A, d, n, k, lda=None):
    lda = n if lda is None else lda
    base = k * lda * n * d
    return [np.asfortranarray(A[base + l * lda * n: base + (l + 1) * lda * n]
                              .reshape(n, lda).T[:n, :]) for l in range(d)]


@pytest.mark.parametrize("variant", ["recur", "alg993"])
def test_batched_golden(golden, variant):
    for c in golden["cases"]:
        if c["kind"] != "batched":
            continue
        d, n, batch = c["d"], c["n"], c["batch"]
        Y = c.arr("Y0").copy()
        oracle.kronmult_batched(d, n, c.arr("A"), c.arr("X"), Y)
        assert rel_err(Y, c.arr(f"Y_{variant}")) <= TOL, c["id"]


def test_batched_dense_known_answer(golden):
    """The reference test's own check (test_kronmult6_batched.cpp:345-406):
    explicit dense kron, max abs err <= 1e-6 -- here much tighter."""
    for c in golden["cases"]:
        if c["kind"] != "batched" or c["n"] ** c["d"] > 729:
            continue
        d, n, batch = c["d"], c["n"], c["batch"]
        L = n ** d
        A, X = c.arr("A"), c.arr("X")
        Y = c.arr("Y0").copy()
        for k in range(batch):
            mats = _square_mats(A, d, n, k)
            oracle.kron_apply(mats, X[k * L:(k + 1) * L], Y[k * L:(k + 1) * L], dense=True)
        assert rel_err(Y, c.arr("Y_recur")) <= TOL, c["id"]
        # and against numpy's kron as a third opinion
        Y2 = c.arr("Y0").copy()
        for k in range(batch):
            mats = _square_mats(A, d, n, k)
            K = mats[0]
            for M in mats[1:]:
                K = np.kron(K, M)
            Y2[k * L:(k + 1) * L] += K @ X[k * L:(k + 1) * L]
        assert rel_err(Y2, c.arr("Y_recur")) <= TOL, c["id"]


def test_pbatched_golden(golden):
    for c in golden["cases"]:
        if c["kind"] != "pbatched":
            continue
        d, n, batch = c["d"], c["n"], c["batch"]
        L = n ** d
        A, X = c.arr("A"), c.arr("X")
        Y = c.arr("Y0").copy()
        ycol = c.arr("y_col")
        ap = [A.ctypes.data + 8 * (k * d + l) * n * n for k in range(batch) for l in range(d)]
        xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
        yp = [Y.ctypes.data + 8 * L * int(ycol[k]) for k in range(batch)]
        oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
        for v in ("recur", "alg993"):
            assert rel_err(Y, c.arr(f"Y_{v}")) <= TOL, (c["id"], v)


def test_xbatched_golden(golden):
    for c in golden["cases"]:
        if c["kind"] != "xbatched":
            continue
        d, n, batch, lda, npool = c["d"], c["n"], c["batch"], c["lda"], c["npool"]
        L = n ** d
        Ap, X = c.arr("Apool"), c.arr("X")
        aidx, xcol, ycol = c.arr("a_idx"), c.arr("x_col"), c.arr("y_col")
        Y = c.arr("Y0").copy()
        ap = [Ap.ctypes.data + 8 * lda * n * (l * npool + int(aidx[k, l]))
              for k in range(batch) for l in range(d)]
        xp = [X.ctypes.data + 8 * L * int(xcol[k]) for k in range(batch)]
        yp = [Y.ctypes.data + 8 * L * int(ycol[k]) for k in range(batch)]
        oracle.kronmult_general(d, [n] * d, [n] * d, ap, [lda] * d, xp, yp)
        for v in ("recur", "alg993"):
            assert rel_err(Y, c.arr(f"Y_{v}")) <= TOL, (c["id"], v)


def test_vbatched_golden(golden):
    for c in golden["cases"]:
        if c["kind"] != "vbatched":
            continue
        d, m, n, batch = c["d"], c["m"], c["n"], c["batch"]
        N, M = int(np.prod(n)), int(np.prod(m))
        A, X = c.arr("A"), c.arr("X")
        aoff, ycol = c.arr("a_off"), c.arr("y_col")
        Y = c.arr("Y0").copy()
        ap = [A.ctypes.data + 8 * int(o) for o in aoff]
        xp = [X.ctypes.data + 8 * N * k for k in range(batch)]
        yp = [Y.ctypes.data + 8 * M * int(ycol[k]) for k in range(batch)]
        oracle.kronmult_general(d, m, n, ap, m, xp, yp)
        assert rel_err(Y, c.arr("Y_recur")) <= TOL, c["id"]


def test_kgemm_golden(golden):
    for c in golden["cases"]:
        if c["kind"] != "kgemm":
            continue
        op, mm, nn, kk, batch = c["op"], c["mm"], c["nn"], c["kk"], c["batch"]
        ldA, ldB, ldC = c["ldA"], c["ldB"], c["ldC"]
        A, B = c.arr("A"), c.arr("B")
        Cm = c.arr("C0").copy()
        ncA = mm if op == "tt" else kk
        ncB = nn if op == "nn" else kk
        ap = [A.ctypes.data + 8 * ldA * ncA * b for b in range(batch)]
        bp = [B.ctypes.data + 8 * ldB * ncB * b for b in range(batch)]
        cp = [Cm.ctypes.data + 8 * ldC * nn * b for b in range(batch)]
        oracle.kgemm_batched(op, mm, nn, kk, c["alpha"], ap, [ldA] * batch, bp, [ldB] * batch,
                             c["beta"], cp, [ldC] * batch)
        assert rel_err(Cm, c.arr("C_ref")) <= 1e-14, c["id"]


def test_kron_flops_golden(golden):
    for f in golden["kron_flops"]:
        assert oracle.kron_flops(f["m"], f["n"]) == f["kron_flops"]


def test_flop_variant_choice():
    # square: forward == backward -> ties go backward (kronm.hpp:89)
    assert not oracle.use_forward([4] * 6, [4] * 6)
    assert oracle.flops_forward([4] * 6, [4] * 6) == 2 * 6 * 4 ** 7
    # shrinking A_1 first is cheaper forward
    assert oracle.use_forward([2, 8, 8], [8, 8, 8])
    assert not oracle.use_forward([8, 8, 2], [8, 8, 8])
