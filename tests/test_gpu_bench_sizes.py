"""GPU parity at the benchmarked sizes: each bench.py workload, built by the
bench's own generators (identical inputs), runs one library step from Y = 0
and is compared with the oracle's restatement over the whole batch.

- config 1: kronmult6_batched n=4, 512 entries;
- config 2: kronmult3_xbatched n=8, 131072 entries with 16-way output
  aliasing, atomic and deterministic segmented modes;
- config 3: kronmult6_batched, 4096 entries, n = 4 and n = 6, FP64 and FP32;
- config 4: the uneven batch of 20000 entries in one plan (the oracle runs
  every (d, shape) group);
- config 5: d=6 n=8 xbatched on a 64-entry slice whose outputs are drawn from
  45 columns (the same aliasing pattern).

The reference checks every result of its own tests the same way
(test_kronmult6_xbatched.cpp:397-560).  Bars: FP64 normwise relative error
<= 1e-13, FP32 <= 1e-5."""
import numpy as np
import pytest

import bench
import kronmult_b200 as kb
import oracle
from tests.golden_cases import rel_err

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-13, "f32": 1e-5}


def _run(torch, wl):
    wl.dY.zero_()
    wl.step()
    torch.cuda.synchronize()
    return wl.dY.double().cpu().numpy()


def _xbatched_oracle(d, n, Apool, aoff, X, xlist, ylist, ny):
    L = n ** d
    Y = np.zeros(L * ny)
    oracle.kronmult_general(d, [n] * d, [n] * d, [Apool.ctypes.data + 8 * int(o) for o in aoff],
                            [n] * d, [X.ctypes.data + 8 * L * int(j) for j in xlist],
                            [Y.ctypes.data + 8 * L * int(i) for i in ylist])
    return Y


@pytest.mark.parametrize("cfg,n,prec", [(1, 4, "f64"), (3, 4, "f64"), (3, 4, "f32"),
                                        (3, 6, "f64"), (3, 6, "f32")])
def test_batched_full_size(gpu_lib, cfg, n, prec):
    import torch

    wl = bench.make_workload(cfg, prec, 0, n)
    wl.setup(torch, kb, "atomic", e2e=False)
    got = _run(torch, wl)
    Y = np.zeros(wl.L * wl.batch)
    oracle.kronmult_batched(wl.d, wl.n, wl.A, wl.X, Y)
    assert rel_err(got, Y) <= TOL[prec]
    assert kb.lib().kron_device_status(1) == 0
    wl.release(torch)


@pytest.mark.parametrize("mode", ["atomic", "segmented"])
def test_xbatched_overlap_full_size(gpu_lib, mode):
    import torch

    wl = bench.make_workload(2, "f64")
    wl.setup(torch, kb, mode)
    got = _run(torch, wl)
    Y = _xbatched_oracle(wl.d, wl.n, wl.Apool, wl.a_offsets(), wl.X, wl.xlist, wl.ylist,
                         wl.nelem)
    assert rel_err(got, Y) <= TOL["f64"]
    assert kb.lib().kron_device_status(1) == 0


def test_uneven_batch_full_size(gpu_lib):
    import torch

    wl = bench.make_workload(4, "f64")
    wl.setup(torch, kb, "atomic")
    got = _run(torch, wl)
    # the oracle over every (d, shape) group of the same entries
    Y = np.zeros(wl.ny)
    groups = {}
    for k in range(wl.batch):
        d = int(wl.shapes[k, 0])
        groups.setdefault(tuple(int(v) for v in wl.shapes[k, :1 + 2 * d]), []).append(k)
    for key, ks in groups.items():
        d = key[0]
        m, nn = list(key[1::2]), list(key[2::2])
        ap = [wl.A.ctypes.data + 8 * int(wl.a_off[6 * k + l]) for k in ks for l in range(d)]
        xp = [wl.X.ctypes.data + 8 * int(wl.x_off[k]) for k in ks]
        yp = [Y.ctypes.data + 8 * int(wl.y_off[k]) for k in ks]
        oracle.kronmult_general(d, m, nn, ap, m, xp, yp)
    assert rel_err(got, Y) <= TOL["f64"]
    assert kb.lib().kron_device_status(1) == 0


def test_config5_slice_with_aliasing(gpu_lib):
    import torch

    wl = bench.XbatchedBig(batch=64, nout=45)
    wl.setup(torch, kb, "atomic")
    assert wl.ndistinct < wl.batch, "outputs alias"
    got = _run(torch, wl)
    X = wl.dX.cpu().numpy()
    Y = _xbatched_oracle(wl.d, wl.n, wl.Apool, wl.a_offsets(), X, np.arange(wl.batch),
                         wl.ylist, wl.nout)
    assert rel_err(got, Y) <= TOL["f64"]
    assert kb.lib().kron_device_status(1) == 0
