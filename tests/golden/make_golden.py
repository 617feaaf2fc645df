"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference KRONMULT CPU implementation (compiled from its own
headers into oracle/_ref/ by ``make -C oracle ref``) on
  * the reference tests' closed-form known-answer inputs
    (test_kronmult6_batched.cpp:117-154, test_kronmult6_xbatched.cpp:185-237,
    test_kgemm_nn_batched.cpp:173-195), and
  * seeded U(-1,1) inputs (numpy PCG64, seeds stated per case),
and stores inputs + the reference's outputs as ``golden.npz`` with a case
index ``golden.json``.  Both reference algorithm variants (recursive and
Alg. 993) are recorded where they are valid; rectangular shapes use the
recursive variant only (the Alg. 993 vbatched workspace is undersized for
them, kronmult_vbatched.hpp:107-135).

Usage:  python tests/golden/make_golden.py      (needs oracle/_ref built)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

SEED0 = 20261203


def closed_form_batched(d, n, batch, lda=None):
    """Reference test inputs (test_kronmult6_batched.cpp:124-150): 1-based
    X(i,k) = (i + (k-1)*Xsize) / (Xsize*batch);
    A(i,j,l,k) = (i + (j-1)n + (l-1)n^2 + (k-1)*batch) / (n^2 d batch)."""
    lda = n if lda is None else lda
    L = n ** d
    X = np.empty(L * batch)
    for k in range(batch):
        i = np.arange(1, L + 1, dtype=np.float64)
        X[k * L:(k + 1) * L] = (i + k * L) / (L * batch)
    A = np.zeros(lda * n * d * batch)
    for k in range(batch):
        for l in range(d):
            for j in range(n):
                for i in range(n):
                    r1 = (i + 1) + j * n + l * n * n + k * batch
                    A[i + j * lda + l * lda * n + k * lda * n * d] = r1 / (n * n * d * batch)
    return A, X


def main():
    refs = {v: oracle.Reference(v) for v in ("recur", "alg993")}
    arrays = {}
    cases = []

    def add(case, **arrs):
        cid = f"c{len(cases):03d}"
        case["id"] = cid
        for k, v in arrs.items():
            arrays[f"{cid}_{k}"] = np.ascontiguousarray(v)
        cases.append(case)

    # ---- batched: closed-form known-answer inputs, both variants ----------
    for d in range(1, 7):
        for n in (1, 2, 3, 4):
            L = n ** d
            batch = 3 if L <= 256 else 1
            A, X = closed_form_batched(d, n, batch)
            Y0 = np.zeros(L * batch)
            outs = {}
            for v, ref in refs.items():
                Y = Y0.copy()
                ref.kronmult_batched(d, n, A.copy(), X.copy(), Y)
                outs[v] = Y
            add({"kind": "batched", "d": d, "n": n, "batch": batch, "inputs": "closed_form"},
                A=A, X=X, Y0=Y0, Y_recur=outs["recur"], Y_alg993=outs["alg993"])

    # ---- batched: seeded U(-1,1), Y0 nonzero (checks accumulation) ---------
    for ci, (d, n, batch) in enumerate([(6, 4, 2), (3, 8, 3), (5, 3, 4), (2, 7, 5), (4, 5, 2),
                                        (1, 9, 6), (6, 2, 8), (3, 5, 4)]):
        rng = np.random.default_rng(SEED0 + 100 + ci)
        L = n ** d
        A = rng.uniform(-1, 1, n * n * d * batch)
        X = rng.uniform(-1, 1, L * batch)
        Y0 = rng.uniform(-1, 1, L * batch)
        outs = {}
        for v, ref in refs.items():
            Y = Y0.copy()
            ref.kronmult_batched(d, n, A.copy(), X.copy(), Y)
            outs[v] = Y
        add({"kind": "batched", "d": d, "n": n, "batch": batch, "inputs": "uniform",
             "seed": SEED0 + 100 + ci},
            A=A, X=X, Y0=Y0, Y_recur=outs["recur"], Y_alg993=outs["alg993"])

    # ---- pbatched: all outputs onto one column (use_overlap_in_Y) ----------
    for ci, (d, n, batch) in enumerate([(1, 4, 5), (2, 3, 6), (3, 4, 4), (4, 3, 3), (5, 2, 6),
                                        (6, 3, 2)]):
        rng = np.random.default_rng(SEED0 + 200 + ci)
        L = n ** d
        A = rng.uniform(-1, 1, n * n * d * batch)
        X = rng.uniform(-1, 1, L * batch)
        ny = 2
        Y0 = rng.uniform(-1, 1, L * ny)
        # entry k writes column (k % 2): two overlapping groups
        y_col = np.array([k % ny for k in range(batch)], dtype=np.int64)
        outs = {}
        for v, ref in refs.items():
            Xc = X.copy()
            Y = Y0.copy()
            W = np.zeros(L * batch)
            xp = [Xc.ctypes.data + 8 * L * k for k in range(batch)]
            yp = [Y.ctypes.data + 8 * L * int(y_col[k]) for k in range(batch)]
            wp = [W.ctypes.data + 8 * L * k for k in range(batch)]
            ref.kronmult_pbatched(d, n, A, xp, yp, wp)
            outs[v] = Y
        add({"kind": "pbatched", "d": d, "n": n, "batch": batch, "ny": ny,
             "seed": SEED0 + 200 + ci},
            A=A, X=X, Y0=Y0, y_col=y_col, Y_recur=outs["recur"], Y_alg993=outs["alg993"])

    # ---- xbatched: A pointers with lda = n+3, overlapping Y, X preserved ---
    for ci, (d, n, batch) in enumerate([(1, 3, 4), (2, 4, 5), (3, 8, 6), (4, 3, 4), (5, 3, 3),
                                        (6, 2, 7), (3, 4, 1)]):
        rng = np.random.default_rng(SEED0 + 300 + ci)
        L = n ** d
        lda = n + 3
        npool = 4
        Apool = rng.uniform(-1, 1, lda * n * npool * d)  # pool of npool matrices per dim
        a_idx = rng.integers(0, npool, size=(batch, d)).astype(np.int64)
        nx = max(1, batch - 1)
        X = rng.uniform(-1, 1, L * nx)
        x_col = rng.integers(0, nx, size=batch).astype(np.int64)
        ny = max(1, (batch + 1) // 2)
        Y0 = rng.uniform(-1, 1, L * ny)
        y_col = rng.integers(0, ny, size=batch).astype(np.int64)
        outs = {}
        for v, ref in refs.items():
            Xc = X.copy()
            Y = Y0.copy()
            W = np.zeros(L * max(2, 2 * batch))
            ap = []
            for k in range(batch):
                for l in range(d):
                    ap.append(Apool.ctypes.data + 8 * lda * n * (l * npool + int(a_idx[k, l])))
            xp = [Xc.ctypes.data + 8 * L * int(x_col[k]) for k in range(batch)]
            yp = [Y.ctypes.data + 8 * L * int(y_col[k]) for k in range(batch)]
            wp = [W.ctypes.data + 8 * L * k for k in range(max(2, 2 * batch))]
            ref.kronmult_xbatched(d, n, ap, lda, xp, yp, wp, 0)
            # with batchCount == 1 the reference skips its X copy and works in
            # X itself (kronmult_xbatched.hpp:112-113), so X is clobbered then
            assert batch == 1 or np.array_equal(Xc, X), "xbatched must preserve X"
            outs[v] = Y
        add({"kind": "xbatched", "d": d, "n": n, "batch": batch, "lda": lda, "npool": npool,
             "nx": nx, "ny": ny, "seed": SEED0 + 300 + ci},
            Apool=Apool, a_idx=a_idx, X=X, x_col=x_col, Y0=Y0, y_col=y_col,
            Y_recur=outs["recur"], Y_alg993=outs["alg993"])

    # ---- vbatched: uniform rectangular shapes (recursive variant only) -----
    shapes = [([3], [2]), ([2, 4], [3, 2]), ([2, 3, 4], [4, 2, 3]), ([3, 2, 2, 3], [2, 3, 2, 2]),
              ([2, 2, 3, 2, 2], [3, 2, 2, 2, 3]), ([2, 3, 2, 2, 2, 2], [2, 2, 2, 3, 2, 2]),
              ([4, 4, 4], [4, 4, 4]), ([8, 2], [2, 8]), ([6, 3, 8], [2, 8, 4])]
    for ci, (m, n) in enumerate(shapes):
        d = len(m)
        rng = np.random.default_rng(SEED0 + 400 + ci)
        batch = 3
        N = int(np.prod(n))
        M = int(np.prod(m))
        A = rng.uniform(-1, 1, sum(mi * ni for mi, ni in zip(m, n)) * batch)
        X = rng.uniform(-1, 1, N * batch)
        Y0 = rng.uniform(-1, 1, M * batch)
        y_col = np.array([0, 1, 0], dtype=np.int64)  # entries 0 and 2 overlap
        Y = Y0.copy()
        Xc = X.copy()
        ap = []
        off = 0
        a_off = []
        for k in range(batch):
            for l in range(d):
                ap.append(A.ctypes.data + 8 * off)
                a_off.append(off)
                off += m[l] * n[l]
        xp = [Xc.ctypes.data + 8 * N * k for k in range(batch)]
        yp = [Y.ctypes.data + 8 * M * int(y_col[k]) for k in range(batch)]
        # generous workspace (the reference sizes per-entry scratch itself)
        W = np.zeros(64 * max(N, M) * batch + 4096)
        refs["recur"].kronmult_vbatched(d, m, n, ap, xp, yp, W)
        assert np.array_equal(Xc, X), "vbatched must preserve X"
        add({"kind": "vbatched", "d": d, "m": m, "n": n, "batch": batch,
             "seed": SEED0 + 400 + ci},
            A=A, a_off=np.array(a_off, dtype=np.int64), X=X, Y0=Y0, y_col=y_col, Y_recur=Y)

    # ---- kgemm_{nn,nt,tt}_batched ------------------------------------------
    for op in ("nn", "nt", "tt"):
        for (mm, nn, kk, batch, alpha, beta, pad, inputs) in [
            (8, 15, 22, 3, 1.3, 1.2, 0, "closed_form"),
            (1, 8, 1, 2, 1.3, 1.2, 0, "closed_form"),
            (29, 36, 8, 2, 1.3, 1.2, 3, "closed_form"),
            (64, 64, 64, 1, 1.3, 1.2, 0, "closed_form"),
            (17, 33, 5, 4, 0.7, 1.0, 2, "uniform"),   # beta == 1 (atomic branch)
            (9, 12, 7, 3, -1.1, 0.0, 1, "uniform"),   # beta == 0 (plain store)
        ]:
            rng = np.random.default_rng(SEED0 + 500 + len(cases))
            nrA, ncA = (kk, mm) if op == "tt" else (mm, kk)
            nrB, ncB = (kk, nn) if op == "nn" else (nn, kk)
            ldA, ldB, ldC = nrA + pad, nrB + pad, mm + pad
            Aall = np.zeros(ldA * ncA * batch)
            Ball = np.zeros(ldB * ncB * batch)
            Call = np.zeros(ldC * nn * batch)
            for b in range(batch):
                Ab = Aall[b * ldA * ncA:(b + 1) * ldA * ncA]
                Bb = Ball[b * ldB * ncB:(b + 1) * ldB * ncB]
                Cb = Call[b * ldC * nn:(b + 1) * ldC * nn]
                for j in range(ncA):
                    for i in range(nrA):
                        Ab[i + j * ldA] = (1.0 + (i + 1) + (j + 1) * nrA + b
                                           if inputs == "closed_form" else rng.uniform(-1, 1))
                for j in range(ncB):
                    for i in range(nrB):
                        Bb[i + j * ldB] = (1.0 / (1.0 + (i + 1) + (j + 1) * nrB + b)
                                           if inputs == "closed_form" else rng.uniform(-1, 1))
                for j in range(nn):
                    for i in range(mm):
                        Cb[i + j * ldC] = 1.0 if inputs == "closed_form" else rng.uniform(-1, 1)
            C0 = Call.copy()
            ap = [Aall.ctypes.data + 8 * ldA * ncA * b for b in range(batch)]
            bp = [Ball.ctypes.data + 8 * ldB * ncB * b for b in range(batch)]
            cp = [Call.ctypes.data + 8 * ldC * nn * b for b in range(batch)]
            refs["recur"].kgemm_batched(op, mm, nn, kk, alpha, ap, [ldA] * batch, bp,
                                        [ldB] * batch, beta, cp, [ldC] * batch)
            add({"kind": "kgemm", "op": op, "mm": mm, "nn": nn, "kk": kk, "batch": batch,
                 "alpha": alpha, "beta": beta, "ldA": ldA, "ldB": ldB, "ldC": ldC,
                 "inputs": inputs},
                A=Aall, B=Ball, C0=C0, C_ref=Call)

    # ---- kron_flops (kroncommon.hpp:154-185) --------------------------------
    flops = []
    for (m, n) in [([4] * 6, [4] * 6), ([8] * 3, [8] * 3), ([2, 3, 4], [4, 3, 2]),
                   ([6, 3, 8], [2, 8, 4]), ([5], [7]), ([2, 8, 3, 6, 4, 2], [3, 2, 8, 2, 6, 4])]:
        flops.append({"m": m, "n": n, "kron_flops": refs["recur"].kron_flops(m, n)})

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference_variants": ["recur", "alg993"],
                   "cases": cases, "kron_flops": flops}, f, indent=1)
    size = os.path.getsize(os.path.join(HERE, "golden.npz"))
    print(f"{len(cases)} cases, golden.npz {size / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
