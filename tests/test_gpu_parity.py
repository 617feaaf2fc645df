"""GPU parity: the CUDA library (through its C ABI) against the reference's
golden outputs and the oracle.  FP64 bar: normwise relative error <= 1e-13
(the summation order differs from the reference's; atomics reorder too)."""
import numpy as np
import pytest

import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err
from tests.gpu_util import dev, host, ptrs

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 1e-5
TOLSPLIT = 1e-12


def _torch():
    import torch

    return torch


# ------------------------------------------------------------------ golden
def test_batched_golden(gpu_lib, golden):
    torch = _torch()
    for c in golden["cases"]:
        if c["kind"] != "batched":
            continue
        d, n = c["d"], c["n"]
        A, X, Y = dev(c.arr("A")), dev(c.arr("X")), dev(c.arr("Y0"))
        X0 = X.clone()
        kb.kronmult_batched(d, n, A, X, Y)
        assert rel_err(host(Y), c.arr("Y_recur")) <= TOL64, c["id"]
        assert rel_err(host(Y), c.arr("Y_alg993")) <= TOL64, c["id"]
        assert torch.equal(X, X0), "X must be preserved"


def test_pbatched_golden(gpu_lib, golden):
    for c in golden["cases"]:
        if c["kind"] != "pbatched":
            continue
        d, n, batch = c["d"], c["n"], c["batch"]
        L = n ** d
        A, X, Y = dev(c.arr("A")), dev(c.arr("X")), dev(c.arr("Y0"))
        pX = ptrs(X, [L * k for k in range(batch)])
        pY = ptrs(Y, [L * int(j) for j in c.arr("y_col")])
        kb.kronmult_pbatched(d, n, A, pX, pY)
        assert rel_err(host(Y), c.arr("Y_recur")) <= TOL64, c["id"]


def _xbatched_inputs(c):
    d, n, batch, lda, npool = c["d"], c["n"], c["batch"], c["lda"], c["npool"]
    L = n ** d
    Ap, X, Y = dev(c.arr("Apool")), dev(c.arr("X")), dev(c.arr("Y0"))
    aidx = c.arr("a_idx")
    pA = ptrs(Ap, [lda * n * (l * npool + int(aidx[k, l])) for k in range(batch)
                   for l in range(d)])
    pX = ptrs(X, [L * int(j) for j in c.arr("x_col")])
    pY = ptrs(Y, [L * int(j) for j in c.arr("y_col")])
    return Ap, X, Y, pA, pX, pY


def test_xbatched_golden(gpu_lib, golden):
    torch = _torch()
    for c in golden["cases"]:
        if c["kind"] != "xbatched":
            continue
        Ap, X, Y, pA, pX, pY = _xbatched_inputs(c)
        X0 = X.clone()
        kb.kronmult_xbatched(c["d"], c["n"], pA, c["lda"], pX, pY)
        assert rel_err(host(Y), c.arr("Y_recur")) <= TOL64, c["id"]
        assert torch.equal(X, X0)


def test_xbatched_golden_segmented(gpu_lib, golden):
    for c in golden["cases"]:
        if c["kind"] != "xbatched":
            continue
        Ap, X, Y, pA, pX, pY = _xbatched_inputs(c)
        seg = kb.Segments(pY)
        assert seg.count == len(set(c.arr("y_col").tolist()))
        kb.kronmult_xbatched_segmented(c["d"], c["n"], pA, c["lda"], pX, pY, seg)
        assert rel_err(host(Y), c.arr("Y_recur")) <= TOL64, c["id"]
        seg.close()


def test_vbatched_golden(gpu_lib, golden):
    for c in golden["cases"]:
        if c["kind"] != "vbatched":
            continue
        m, n, batch = c["m"], c["n"], c["batch"]
        N, M = int(np.prod(n)), int(np.prod(m))
        A, X, Y = dev(c.arr("A")), dev(c.arr("X")), dev(c.arr("Y0"))
        pA = ptrs(A, c.arr("a_off"))
        pX = ptrs(X, [N * k for k in range(batch)])
        pY = ptrs(Y, [M * int(j) for j in c.arr("y_col")])
        kb.kronmult_vbatched(m, n, pA, pX, pY)
        assert rel_err(host(Y), c.arr("Y_recur")) <= TOL64, c["id"]


def test_kgemm_golden(gpu_lib, golden):
    torch = _torch()
    for c in golden["cases"]:
        if c["kind"] != "kgemm":
            continue
        op, mm, nn, kk, batch = c["op"], c["mm"], c["nn"], c["kk"], c["batch"]
        ldA, ldB, ldC = c["ldA"], c["ldB"], c["ldC"]
        A, B, Cm = dev(c.arr("A")), dev(c.arr("B")), dev(c.arr("C0"))
        ncA = mm if op == "tt" else kk
        ncB = nn if op == "nn" else kk
        pA = ptrs(A, [ldA * ncA * b for b in range(batch)])
        pB = ptrs(B, [ldB * ncB * b for b in range(batch)])
        pC = ptrs(Cm, [ldC * nn * b for b in range(batch)])
        li = lambda v: torch.full((batch,), v, dtype=torch.int32, device="cuda")  # noqa: E731
        kb.kgemm_batched(op, mm, nn, kk, c["alpha"], pA, li(ldA), pB, li(ldB), c["beta"], pC,
                         li(ldC))
        assert rel_err(host(Cm), c.arr("C_ref")) <= 1e-14, c["id"]


# ------------------------------------------------------------- vs oracle
def _rand_batched(d, n, batch, seed):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, n * n * d * batch)
    X = rng.uniform(-1, 1, n ** d * batch)
    Y0 = rng.uniform(-1, 1, n ** d * batch)
    return A, X, Y0


@pytest.mark.parametrize("d,n,batch", [
    (6, 4, 64),   # config-1 shape, compile-time kernel
    (6, 5, 6),    # 125 KB vector: on chip without merge buffer
    (6, 6, 3),    # 373 KB: two-phase workspace path
    (5, 8, 2),    # 262 KB: two-phase
    (4, 9, 3),    # n outside the compile-time set: runtime kernel
    (2, 16, 5),
    (3, 1, 4),    # n == 1
    (1, 7, 9),    # d == 1 (kgemm_nn in the reference, kronmult1.hpp:38-51)
    (3, 8, 40),
    (6, 3, 33),
])
def test_batched_vs_oracle(gpu_lib, d, n, batch):
    A, X, Y0 = _rand_batched(d, n, batch, 1000 + 7 * d + n)
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    dA, dX, dY = dev(A), dev(X), dev(Y0)
    need = kb.lib().kron_batched_workspace_bytes(d, n, batch)
    W = None
    if need:
        W = _torch().empty(need // 8, dtype=_torch().float64, device="cuda")
    kb.kronmult_batched(d, n, dA, dX, dY, W)
    assert rel_err(host(dY), Yref) <= TOL64


def test_batched_needs_workspace(gpu_lib):
    """n^d beyond one block's shared memory and beyond a two-block cluster's
    (d = 6, n = 7: 941 KB) needs the caller's W; d = 6, n = 6 no longer does
    (W in the cluster's shared memory, tests/test_gpu_dsm.py)."""
    d, n, batch = 6, 7, 2
    A, X, Y0 = _rand_batched(d, n, batch, 3)
    assert kb.lib().kron_batched_workspace_bytes(d, n, batch) > 0
    with pytest.raises(kb.KronError) as ei:
        kb.kronmult_batched(d, n, dev(A), dev(X), dev(Y0), None)
    assert ei.value.status == 2


def test_unaligned_operands(gpu_lib):
    """Vectors starting 8 bytes off a 16-byte boundary take the scalar path."""
    torch = _torch()
    d, n, batch = 3, 4, 5
    A, X, Y0 = _rand_batched(d, n, batch, 11)
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    dA = dev(np.concatenate([[0.0], A]))[1:]
    dX = dev(np.concatenate([[0.0], X]))[1:]
    dY = dev(np.concatenate([[0.0], Y0]))[1:]
    kb.kronmult_batched(d, n, dA, dX, dY)
    assert rel_err(host(dY), Yref) <= TOL64


def _xbatched_problem(nelem, nnb, d, n, npool, seed):
    """Element grid: entry (i, t) adds kron(A..) X_j into Y_i, j = self or a
    random neighbour (the overlapping-output workload, scaled down)."""
    rng = np.random.default_rng(seed)
    L = n ** d
    Apool = rng.standard_normal(n * n * npool * d) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * nelem)
    Y0 = rng.uniform(-1, 1, L * nelem)
    ylist, xlist = [], []
    for i in range(nelem):
        nb = rng.choice(np.delete(np.arange(nelem), i), size=nnb - 1, replace=False)
        for j in [i] + list(nb):
            ylist.append(i)
            xlist.append(int(j))
    batch = len(ylist)
    aidx = rng.integers(0, npool, size=(batch, d))
    return Apool, X, Y0, np.array(ylist), np.array(xlist), aidx


def test_xbatched_overlap_atomic_and_segmented(gpu_lib):
    torch = _torch()
    d, n, npool = 3, 8, 64
    Apool, X, Y0, yl, xl, aidx = _xbatched_problem(96, 16, d, n, npool, 77)
    L, batch = n ** d, len(yl)
    # oracle
    Yref = Y0.copy()
    ap = [Apool.ctypes.data + 8 * n * n * (l * npool + int(aidx[k, l])) for k in range(batch)
          for l in range(d)]
    xp = [X.ctypes.data + 8 * L * int(j) for j in xl]
    yp = [Yref.ctypes.data + 8 * L * int(i) for i in yl]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)

    dA, dX = dev(Apool), dev(X)
    pA = ptrs(dA, [n * n * (l * npool + int(aidx[k, l])) for k in range(batch) for l in range(d)])
    pX = ptrs(dX, [L * int(j) for j in xl])
    # atomic (reference semantics)
    dY = dev(Y0)
    pY = ptrs(dY, [L * int(i) for i in yl])
    kb.kronmult_xbatched(d, n, pA, n, pX, pY)
    assert rel_err(host(dY), Yref) <= TOL64
    # deterministic: same result bitwise on every run
    seg = kb.Segments(pY)
    assert seg.count == 96
    dY2 = dev(Y0)
    pY2 = ptrs(dY2, [L * int(i) for i in yl])
    seg2 = kb.Segments(pY2)
    Y0d = dev(Y0)
    outs = []
    for _ in range(3):
        dY2.copy_(Y0d)
        kb.kronmult_xbatched_segmented(d, n, pA, n, pX, pY2, seg2)
        outs.append(host(dY2))
    assert rel_err(outs[0], Yref) <= TOL64
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    # shuffled entry order: the segmented sum order follows the plan
    perm = np.random.default_rng(1).permutation(batch)
    dY3 = dev(Y0)
    pY3 = ptrs(dY3, [L * int(yl[k]) for k in perm])
    pX3 = ptrs(dX, [L * int(xl[k]) for k in perm])
    pA3 = ptrs(dA, [n * n * (l * npool + int(aidx[k, l])) for k in perm for l in range(d)])
    seg3 = kb.Segments(pY3)
    kb.kronmult_xbatched_segmented(d, n, pA3, n, pX3, pY3, seg3)
    assert rel_err(host(dY3), Yref) <= TOL64
    seg.close()
    seg2.close()
    seg3.close()
    del torch


def test_pbatched_segmented(gpu_lib):
    d, n, batch = 4, 5, 24
    A, X, Y0 = _rand_batched(d, n, batch, 91)
    L = n ** d
    ycol = np.arange(batch) % 5
    Yref = Y0.copy()
    ap = [A.ctypes.data + 8 * (k * d + l) * n * n for k in range(batch) for l in range(d)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * L * int(j) for j in ycol]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
    dA, dX, dY = dev(A), dev(X), dev(Y0)
    pX = ptrs(dX, [L * k for k in range(batch)])
    pY = ptrs(dY, [L * int(j) for j in ycol])
    seg = kb.Segments(pY)
    kb.kronmult_pbatched_segmented(d, n, dA, pX, pY, seg)
    assert rel_err(host(dY), Yref) <= TOL64
    seg.close()


def test_large_vectors_overlapping_outputs(gpu_lib):
    """xbatched with n^d beyond shared memory: two-phase path through pW,
    atomic and segmented."""
    torch = _torch()
    d, n = 6, 6
    batch, ny = 4, 2
    rng = np.random.default_rng(5)
    L = n ** d
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * ny)
    ycol = [0, 1, 0, 1]
    Yref = Y0.copy()
    ap = [A.ctypes.data + 8 * (k * d + l) * n * n for k in range(batch) for l in range(d)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * L * j for j in ycol]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
    dA, dX = dev(A), dev(X)
    pA = ptrs(dA, [(k * d + l) * n * n for k in range(batch) for l in range(d)])
    pX = ptrs(dX, [L * k for k in range(batch)])
    Wbuf = torch.empty(L * batch, dtype=torch.float64, device="cuda")
    pW = ptrs(Wbuf, [L * k for k in range(batch)])
    dY = dev(Y0)
    pY = ptrs(dY, [L * j for j in ycol])
    kb.kronmult_xbatched(d, n, pA, n, pX, pY, pW)
    assert rel_err(host(dY), Yref) <= TOL64
    dY2 = dev(Y0)
    pY2 = ptrs(dY2, [L * j for j in ycol])
    seg = kb.Segments(pY2)
    kb.kronmult_xbatched_segmented(d, n, pA, n, pX, pY2, seg, pW)
    assert rel_err(host(dY2), Yref) <= TOL64
    seg.close()


@pytest.mark.parametrize("d,n,layout,offset", [
    (6, 4, "pbatched", 0), (6, 4, "pbatched", 1), (6, 4, "xbatched", 0), (5, 4, "xbatched", 1),
    (6, 3, "pbatched", 0), (4, 5, "xbatched", 0), (5, 5, "pbatched", 1), (5, 5, "batched", 0),
])
def test_pipelined_layouts(gpu_lib, d, n, layout, offset):
    """The TMA-pipelined kernel (n in 3..5, 4-64 KB vectors) in every layout;
    offset=1 shifts every vector by 8 bytes so the bulk-copy alignment
    fallback runs; outputs alias pairwise in the pointer layouts."""
    rng = np.random.default_rng(900 + 10 * d + n + offset)
    L, batch = n ** d, 37
    A = rng.uniform(-1, 1, n * n * d * batch + offset)
    X = rng.uniform(-1, 1, L * batch + offset)
    ny = batch if layout == "batched" else (batch + 1) // 2
    Y0 = rng.uniform(-1, 1, L * ny + offset)
    ycol = np.arange(batch) if layout == "batched" else np.arange(batch) // 2
    Yref = Y0.copy()
    lda = n + 2 if layout == "xbatched" else n
    Ax = np.zeros(lda * n * d * batch + offset)
    for k in range(batch):
        for l in range(d):
            blk = A[offset + (k * d + l) * n * n: offset + (k * d + l + 1) * n * n].reshape(n, n)
            Ax[offset + (k * d + l) * lda * n: offset + (k * d + l + 1) * lda * n] = \
                np.pad(blk, ((0, 0), (0, lda - n))).reshape(-1)
    src = Ax if layout == "xbatched" else A
    ap = [src.ctypes.data + 8 * (offset + (k * d + l) * lda * n) for k in range(batch)
          for l in range(d)]
    xp = [X.ctypes.data + 8 * (offset + L * k) for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * (offset + L * int(j)) for j in ycol]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [lda] * d, xp, yp)
    dA, dX, dY = dev(src), dev(X), dev(Y0)
    if layout == "batched":
        assert offset == 0
        kb.kronmult_batched(d, n, dA, dX, dY)
    else:
        pX = ptrs(dX, [offset + L * k for k in range(batch)])
        pY = ptrs(dY, [offset + L * int(j) for j in ycol])
        if layout == "pbatched":
            kb.kronmult_pbatched(d, n, dA[offset:], pX, pY)
        else:
            pA = ptrs(dA, [offset + (k * d + l) * lda * n for k in range(batch) for l in range(d)])
            kb.kronmult_xbatched(d, n, pA, lda, pX, pY)
    assert rel_err(host(dY), Yref) <= TOL64
    assert kb.lib().kron_device_status(1) == 0


@pytest.mark.parametrize("d,n,prec,batch", [
    (6, 3, "f64", 1200), (5, 5, "f64", 1200), (4, 5, "f64", 1200), (6, 4, "f64", 1200),
    (5, 4, "f64", 1200), (6, 4, "f32", 1800), (5, 4, "f32", 1800), (5, 5, "f32", 1800),
    (6, 5, "f32", 900),
])
def test_pipelined_every_stage(gpu_lib, d, n, prec, batch):
    """Enough entries that every block of the pipelined kernel cycles
    through all of its stages (odd vector lengths included, whose stage
    slots are padded to 16 bytes), in FP64 and in FP32."""
    torch = _torch()
    rng = np.random.default_rng(1700 + 10 * d + n)
    L = n ** d
    A = rng.uniform(-1, 1, n * n * d * batch)
    X = rng.uniform(-1, 1, L * batch)
    Y0 = rng.uniform(-1, 1, L * batch)
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    if prec == "f64":
        dY = dev(Y0)
        kb.kronmult_batched(d, n, dev(A), dev(X), dY)
        tol = TOL64
    else:
        dY = dev(Y0, torch.float32)
        kb.kronmult_batched_f32(d, n, dev(A, torch.float32), dev(X, torch.float32), dY, None)
        tol = TOL32
    assert rel_err(host(dY).astype(np.float64), Yref) <= tol
    assert kb.lib().kron_device_status(1) == 0


@pytest.mark.parametrize("d,n,batch,prec,layout", [
    (6, 7, 3, "f64", "batched"), (6, 8, 2, "f64", "batched"), (5, 8, 5, "f64", "pbatched"),
    (6, 8, 3, "f64", "xbatched"), (6, 7, 2, "f32", "batched"), (6, 8, 2, "f32", "batched"),
    (6, 6, 9, "f64", "pbatched"),
])
def test_cluster_two_phase(gpu_lib, d, n, batch, prec, layout):
    """Vectors beyond shared memory: one thread-block cluster per entry,
    phase 1 (trailing modes, warp per block; FP64 tensor cores for n = 8),
    phase 2 (leading modes on column tiles).  Pointer layouts alias
    outputs pairwise and give fewer W slots than entries for xbatched."""
    torch = _torch()
    rng = np.random.default_rng(77 + 10 * d + n + batch)
    L = n ** d
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, L * batch)
    ny = batch if layout == "batched" else (batch + 1) // 2
    Y0 = rng.uniform(-1, 1, L * ny)
    ycol = np.arange(batch) if layout == "batched" else np.arange(batch) // 2
    Yref = Y0.copy()
    ap = [A.ctypes.data + 8 * (k * d + l) * n * n for k in range(batch) for l in range(d)]
    xp = [X.ctypes.data + 8 * L * k for k in range(batch)]
    yp = [Yref.ctypes.data + 8 * L * int(j) for j in ycol]
    oracle.kronmult_general(d, [n] * d, [n] * d, ap, [n] * d, xp, yp)
    dt = torch.float32 if prec == "f32" else torch.float64
    dA, dX, dY = dev(A, dt), dev(X, dt), dev(Y0, dt)
    es = 4 if prec == "f32" else 8
    if layout == "batched":
        W = torch.empty(L * batch, dtype=dt, device="cuda")
        if prec == "f32":
            kb.kronmult_batched_f32(d, n, dA, dX, dY, W)
        else:
            kb.kronmult_batched(d, n, dA, dX, dY, W)
    else:
        nw = batch if layout == "pbatched" else 2  # xbatched: 2*subbatch pointers
        Wb = torch.empty(L * nw, dtype=dt, device="cuda")
        pW = ptrs(Wb, [L * k for k in range(nw)], es)
        pX = ptrs(dX, [L * k for k in range(batch)], es)
        pY = ptrs(dY, [L * int(j) for j in ycol], es)
        if layout == "pbatched":
            kb.kronmult_pbatched(d, n, dA, pX, pY, pW)
        else:
            pA = ptrs(dA, [(k * d + l) * n * n for k in range(batch) for l in range(d)], es)
            kb.kronmult_xbatched(d, n, pA, n, pX, pY, pW, subbatch=1)
    tol = TOL32 if prec == "f32" else TOL64
    assert rel_err(host(dY).astype(np.float64), Yref) <= tol
    assert kb.lib().kron_device_status(1) == 0


# ------------------------------------------------------------- precision
@pytest.mark.parametrize("d,n,batch", [(6, 4, 32), (3, 8, 16), (6, 6, 2), (2, 5, 7)])
def test_fp32_and_split(gpu_lib, d, n, batch):
    torch = _torch()
    rng = np.random.default_rng(300 + d * 10 + n)
    A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
    X = rng.uniform(-1, 1, n ** d * batch)
    Yref = np.zeros(n ** d * batch)
    oracle.kronmult_batched(d, n, A, X, Yref)
    need = kb.lib().kron_batched_workspace_bytes(d, n, batch)
    # FP32 storage / FP32 accumulation
    Y32 = torch.zeros(n ** d * batch, dtype=torch.float32, device="cuda")
    W32 = torch.empty(max(1, need // 8), dtype=torch.float32, device="cuda") if need else None
    kb.kronmult_batched_f32(d, n, dev(A, torch.float32), dev(X, torch.float32), Y32, W32)
    e32 = rel_err(host(Y32).astype(np.float64), Yref)
    assert e32 <= TOL32, e32
    # split hi+lo FP32 arithmetic on FP64 storage
    Ys = torch.zeros(n ** d * batch, dtype=torch.float64, device="cuda")
    Ws = torch.empty(max(1, need // 8), dtype=torch.float64, device="cuda") if need else None
    kb.kronmult_batched_split(d, n, dev(A), dev(X), Ys, Ws)
    es = rel_err(host(Ys), Yref)
    assert es <= TOLSPLIT, es


# ------------------------------------------------------------- uneven batch
def _uneven(nentries, seed, dmax=6, sizes=(2, 3, 4, 6, 8)):
    rng = np.random.default_rng(seed)
    shapes = np.zeros((nentries, 13), dtype=np.int32)
    for k in range(nentries):
        d = int(rng.integers(1, dmax + 1))
        shapes[k, 0] = d
        for l in range(d):
            shapes[k, 1 + 2 * l] = rng.choice(sizes)
            shapes[k, 2 + 2 * l] = rng.choice(sizes)
    return shapes


def test_vplan_uneven(gpu_lib):
    torch = _torch()
    shapes = _uneven(120, 2024, dmax=5)
    # include a few vectors beyond shared memory
    big = np.array([[6, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 6],
                    [5, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 0, 0],
                    [6, 2, 8, 8, 8, 3, 8, 8, 8, 8, 2, 8, 8]], dtype=np.int32)
    shapes = np.concatenate([shapes, big])
    rng = np.random.default_rng(7)
    nent = shapes.shape[0]
    a_off, x_off, y_off = [], [], []
    na = nx = ny = 0
    for k in range(nent):
        d = shapes[k, 0]
        m = shapes[k, 1:1 + 2 * d:2]
        n = shapes[k, 2:2 + 2 * d:2]
        for l in range(6):
            a_off.append(na)
            if l < d:
                na += int(m[l] * n[l])
        x_off.append(nx)
        nx += int(np.prod(n))
        # every 3rd entry shares the previous output when shapes agree
        if k > 0 and k % 3 == 0 and shapes[k - 1, 0] == d and \
                np.prod(shapes[k - 1, 1:1 + 2 * d:2]) == np.prod(m):
            y_off.append(y_off[-1])
        else:
            y_off.append(ny)
            ny += int(np.prod(m))
    A = rng.uniform(-1, 1, na)
    X = rng.uniform(-1, 1, nx)
    Y0 = rng.uniform(-1, 1, ny)
    Yref = Y0.copy()
    for k in range(nent):
        d = shapes[k, 0]
        m = [int(v) for v in shapes[k, 1:1 + 2 * d:2]]
        n = [int(v) for v in shapes[k, 2:2 + 2 * d:2]]
        ap = [A.ctypes.data + 8 * a_off[6 * k + l] for l in range(d)]
        oracle.kronmult_general(d, m, n, ap, m, [X.ctypes.data + 8 * x_off[k]],
                                [Yref.ctypes.data + 8 * y_off[k]])
    plan = kb.VPlan(shapes)
    dA, dX, dY = dev(A), dev(X), dev(Y0)
    pA = ptrs(dA, a_off)
    pX = ptrs(dX, x_off)
    pY = ptrs(dY, y_off)
    W = None
    if plan.workspace_bytes:
        W = torch.empty(plan.workspace_bytes // 8, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan.execute(pA, pX, pY, W, stream=s)   # captured into a graph
    s.synchronize()
    assert rel_err(host(dY), Yref) <= TOL64
    # replay (graph reuse) accumulates a second time
    with torch.cuda.stream(s):
        plan.execute(pA, pX, pY, W, stream=s)
    s.synchronize()
    Yref2 = Yref + (Yref - Y0)
    assert rel_err(host(dY), Yref2) <= TOL64
    plan.close()


# -------------------------------------------------- reference C++ signature
def test_reference_signature_cpp_linkage(gpu_lib):
    """Call the mangled C++ symbol kronmult6_batched(int, double const*, ...)
    exactly as a relinked reference caller would (legacy default stream)."""
    import ctypes as C

    torch = _torch()
    lib = C.CDLL(kb.LIB_PATH)
    f = lib["_Z17kronmult6_batchediPKdPdS1_S1_i"]
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    f.restype = None
    d, n, batch = 6, 4, 8
    A, X, Y0 = _rand_batched(d, n, batch, 55)
    Yref = Y0.copy()
    oracle.kronmult_batched(d, n, A, X, Yref)
    dA, dX, dY, dW = dev(A), dev(X), dev(Y0), dev(np.zeros_like(X))
    torch.cuda.synchronize()
    f(n, dA.data_ptr(), dX.data_ptr(), dY.data_ptr(), dW.data_ptr(), batch)
    torch.cuda.synchronize()
    assert kb.lib().kron_get_last_status() == 0
    assert rel_err(host(dY), Yref) <= TOL64
