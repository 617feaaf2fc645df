#!/usr/bin/env python
"""Benchmark of the batched Kronecker matvec on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 1..5] [--n N] [--precision f64|f32|split]
                    [--mode atomic|segmented]

Default workload (the headline): the precision sweep's largest case,
kronmult6_batched with d=6, n=6, FP64, batchCount=4096 (46656-element
vectors, 4.59 GB of algorithmic traffic per step), A ~ N(0,1)/sqrt(6),
X ~ U(-1,1), Y from zero.  Its line also carries
  - max_rel_err: the result of one step against the reference's own
    OpenMP output on the same inputs, over the whole batch;
  - comparison: FP32 and split (hi+lo FP32 arithmetic on FP64 data) legs at
    n = 4 and n = 6 plus the FP64 leg at n = 4, each with its time, HBM GB/s
    and error against the reference's FP64 output.
Other --config values: 1 kronmult6_batched n=4 batch 512; 2 kronmult3_xbatched
n=8 over 8192 elements x 16 couplings (131072 entries, overlapping outputs);
3 the precision sweep (--n 4 or 6, --precision); 4 uneven batch of 20000
entries; 5 d=6 n=8 batch 1024 with shared outputs; 6 kgemm_nn_batched
64x64x64, batch 32768.  All data is synthetic
(seeded numpy PCG64); the reference publishes no dataset.

One step = one call of the library over the whole batch with inputs resident
in HBM.  Steps are timed one by one with CUDA events on the launching stream
and L2 is flushed (256 MB write) between timed steps, outside the events.
Multi-GPU: replicas (each rank runs the whole workload; no collective on the
data path), barrier + max over ranks.

Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20261203
METRIC = "kronmult GFLOP/s + HBM GB/s vs roofline; FP32/split vs FP64 speedup at stated err"


# ---------------------------------------------------------------- workloads
E2E_CHUNKS = 16  # 16 chunks measured 61.3 ms per headline e2e step against 63.2 with 8


def max_rel_err(torch, y, yref):
    """max |y - yref| / max |yref| over the whole output (FP64)."""
    den = yref.abs().max().item()
    return (y.double() - yref).abs().max().item() / (den if den > 0 else 1.0)


def errors_vs(y, yref):
    """Errors of a result against a reference output (host arrays): the
    normwise relative error max |y - yref| / max |yref|, and the reference
    tests' own measure, the largest absolute error max |y - yref|
    (test_kronmult6_batched.cpp:393-394)."""
    y = np.asarray(y, dtype=np.float64)
    yref = np.asarray(yref, dtype=np.float64)
    diff = float(np.abs(y - yref).max()) if y.size else 0.0
    den = float(np.abs(yref).max()) if yref.size else 0.0
    return {"max_rel_err": diff / (den if den > 0 else 1.0), "max_abs_err": diff}


class Workload:
    name = ""
    dtype = "f64"
    launches_per_step = 1
    e2e_pipeline = None  # description of a chunked end-to-end step, if any
    _yref = None

    def reference_y(self):
        """The reference's own output for the whole batch, Y from zero
        (oracle/_ref: the reference's OpenMP build, recursive variant); cached."""
        if self._yref is None:
            import oracle

            ref = oracle.Reference("recur")
            self.cpu_setup(self.batch)
            self.cpu_step(ref)
            self._yref = self.cY.copy()
        return self._yref

    def check(self, torch, yref=None):
        """Errors of one library step (Y from zero) against the reference's
        output on the same inputs."""
        yref = self.reference_y() if yref is None else yref
        self.dY.zero_()
        self.step()
        torch.cuda.synchronize()
        return errors_vs(self.dY.double().cpu().numpy(), yref)

    def flops(self) -> float:
        raise NotImplementedError

    def alg_bytes(self) -> float:
        raise NotImplementedError

    def run_pipeline(self, torch, pre_h2d, chunks):
        """Host <-> device copies overlapped with the library calls: `pre_h2d`
        (dst, src) pairs first, then per chunk its uploads, its call and its
        downloads, on three streams ordered by events (uploads, calls and
        downloads of different chunks overlap; PCIe runs both directions at
        once).  Ends with the current stream waiting for all three."""
        if not hasattr(self, "_streams"):
            self._streams = [torch.cuda.Stream() for _ in range(3)]
        s_in, s_run, s_out = self._streams
        cur = torch.cuda.current_stream()
        for s in self._streams:
            s.wait_stream(cur)
        with torch.cuda.stream(s_in):
            for dst, src in pre_h2d:
                dst.copy_(src, non_blocking=True)
        for h2d, run, d2h in chunks:
            with torch.cuda.stream(s_in):
                for dst, src in h2d:
                    dst.copy_(src, non_blocking=True)
            e_in = torch.cuda.Event()
            e_in.record(s_in)
            s_run.wait_event(e_in)
            run(s_run)
            e_run = torch.cuda.Event()
            e_run.record(s_run)
            s_out.wait_event(e_run)
            with torch.cuda.stream(s_out):
                for dst, src in d2h:
                    dst.copy_(src, non_blocking=True)
        for s in self._streams:
            cur.wait_stream(s)


class XbatchedOverlap(Workload):
    """kronmult3_xbatched d=3 n=8, 8192 elements x 16 couplings (131072 entries)."""

    def __init__(self, nelem=8192, ncoup=16, d=3, n=8, npool=64, seed=SEED + 1):
        rng = np.random.default_rng(seed)
        self.d, self.n, self.npool, self.nelem = d, n, npool, nelem
        self.L = n ** d
        self.Apool = rng.standard_normal(n * n * npool * d) / np.sqrt(n)
        ylist = np.repeat(np.arange(nelem), ncoup)
        xlist = np.empty(nelem * ncoup, dtype=np.int64)
        for i in range(nelem):
            nb = rng.choice(nelem - 1, size=ncoup - 1, replace=False)
            nb = nb + (nb >= i)  # skip self
            xlist[i * ncoup] = i
            xlist[i * ncoup + 1:(i + 1) * ncoup] = nb
        self.ylist, self.xlist = ylist, xlist
        self.batch = len(ylist)
        self.aidx = rng.integers(0, npool, size=(self.batch, d))
        self.X = rng.uniform(-1, 1, self.L * nelem)
        self.name = (f"kronmult{d}_xbatched n={n} FP64, {nelem} elements x {ncoup} couplings "
                     f"= {self.batch} entries, A pool {npool}/dim")

    def flops(self):
        return float(self.batch) * 2 * self.d * self.n ** (self.d + 1)

    def alg_bytes(self):
        # distinct X read once, distinct Y read+written once, A pool once
        return 8.0 * (self.L * self.nelem + 2 * self.L * self.nelem + self.Apool.size)

    def a_offsets(self):
        n, d, npool = self.n, self.d, self.npool
        l = np.arange(d)[None, :]
        return (n * n * (l * npool + self.aidx)).reshape(-1)

    # -- GPU
    def setup(self, torch, kb, mode):
        dev = torch.device("cuda")
        self.kb = kb
        self.mode = mode
        self.dA = torch.from_numpy(self.Apool).to(dev)
        self.dX = torch.from_numpy(self.X).to(dev)
        self.dY = torch.zeros(self.L * self.nelem, dtype=torch.float64, device=dev)
        self.pA = (self.dA.data_ptr() + 8 * torch.from_numpy(self.a_offsets())).to(dev)
        self.pX = (self.dX.data_ptr() + 8 * self.L * torch.from_numpy(self.xlist)).to(dev)
        self.pY = (self.dY.data_ptr() + 8 * self.L * torch.from_numpy(self.ylist)).to(dev)
        self.seg = kb.Segments(self.pY) if mode == "segmented" else None
        # e2e: pinned host copies of every input of the call.  Atomic mode
        # uploads the element grid as int32 index lists and builds the pointer
        # arrays on the device (kron_build_pointers_async); segmented mode
        # uploads the pointer arrays its plan was made for.
        ilists = dict(alist=torch.from_numpy((self.a_offsets() // (self.n * self.n))
                                             .astype(np.int32)),
                      xlist=torch.from_numpy(self.xlist.astype(np.int32)),
                      ylist=torch.from_numpy(self.ylist.astype(np.int32)))
        host_in = dict(A=self.dA, X=self.dX, Y=self.dY)
        if mode == "segmented":
            host_in.update(pA=self.pA, pX=self.pX, pY=self.pY)
        self.h = {k: v.cpu().pin_memory() for k, v in host_in.items()}
        if mode != "segmented":
            self.h.update({k: v.pin_memory() for k, v in ilists.items()})
            self.dlist = {k: v.to(dev) for k, v in ilists.items()}
        self.hYout = torch.empty_like(self.h["Y"]).pin_memory()
        self.h2d_bytes = sum(v.numel() * v.element_size() for v in self.h.values())
        self.d2h_bytes = self.hYout.numel() * 8
        if mode != "segmented":
            self.e2e_pipeline = (f"{E2E_CHUNKS} chunks of whole output elements; int32 index "
                                 "lists up, pointer arrays built on the device; uploads, "
                                 "calls and downloads overlapped on 3 streams")

    def step(self):
        if self.seg is not None:
            self.kb.kronmult_xbatched_segmented(self.d, self.n, self.pA, self.n, self.pX,
                                                self.pY, self.seg)
        else:
            self.kb.kronmult_xbatched(self.d, self.n, self.pA, self.n, self.pX, self.pY)

    def e2e_step(self):
        # host -> device (pinned, async), the library call(s), device -> host
        # of Y.  Atomic mode: entries are ordered by output element, so the
        # batch splits into chunks with disjoint Y ranges; X and the A pool
        # go first, then per chunk its index lists and Y columns, the pointer
        # build and the call, and its Y columns back -- overlapped.
        import torch

        h = self.h
        if self.seg is not None:
            for k in ("A", "X", "Y", "pA", "pX", "pY"):
                getattr(self, "d" + k if k in ("A", "X", "Y") else k).copy_(h[k],
                                                                           non_blocking=True)
            self.step()
            self.hYout.copy_(self.dY, non_blocking=True)
            return
        E = self.nelem // E2E_CHUNKS * (self.batch // self.nelem)  # entries per chunk
        L, d = self.L, self.d
        chunks = []
        for c in range(E2E_CHUNKS):
            e0, e1 = c * E, (c + 1) * E if c < E2E_CHUNKS - 1 else self.batch
            y0, y1 = self.ylist[e0] * L, (self.ylist[e1 - 1] + 1) * L
            dl = self.dlist
            h2d = [(dl["alist"][e0 * d:e1 * d], h["alist"][e0 * d:e1 * d]),
                   (dl["xlist"][e0:e1], h["xlist"][e0:e1]), (dl["ylist"][e0:e1], h["ylist"][e0:e1]),
                   (self.dY[y0:y1], h["Y"][y0:y1])]

            def run(s, e0=e0, e1=e1, dl=dl):
                pA = self.pA[e0 * d:e1 * d]
                pX, pY = self.pX[e0:e1], self.pY[e0:e1]
                nn = self.n * self.n
                rc = self.kb.lib().kron_build_pointers_async(
                    d, e1 - e0, self.dA.data_ptr(), nn, dl["alist"][e0 * d:e1 * d].data_ptr(),
                    self.dX.data_ptr(), L, dl["xlist"][e0:e1].data_ptr(), self.dY.data_ptr(), L,
                    dl["ylist"][e0:e1].data_ptr(), pA.data_ptr(), pX.data_ptr(), pY.data_ptr(),
                    s.cuda_stream)
                if rc != 0:
                    raise RuntimeError(f"kron_build_pointers_async failed: {rc}")
                self.kb.kronmult_xbatched(d, self.n, pA, self.n, pX, pY, stream=s)

            chunks.append((h2d, run, [(self.hYout[y0:y1], self.dY[y0:y1])]))
        self.run_pipeline(torch, [(self.dX, h["X"]), (self.dA, h["A"])], chunks)

    # -- CPU reference (OpenMP build of the reference's own kronmult3_xbatched)
    def cpu_setup(self, sample_entries):
        self.cs = min(self.batch, sample_entries)
        self.cX = self.X.copy()
        self.cY = np.zeros(self.L * self.nelem)
        self.cW = np.zeros(self.L * self.cs)
        base_a = self.Apool.ctypes.data
        self.c_ap = (base_a + 8 * self.a_offsets()[: self.cs * self.d]).astype(np.uint64)
        self.c_xp = (self.cX.ctypes.data + 8 * self.L * self.xlist[: self.cs]).astype(np.uint64)
        self.c_yp = (self.cY.ctypes.data + 8 * self.L * self.ylist[: self.cs]).astype(np.uint64)
        self.c_wp = (self.cW.ctypes.data + 8 * self.L * np.arange(self.cs)).astype(np.uint64)
        return self.cs

    def cpu_step(self, ref):
        ref.kronmult_xbatched(self.d, self.n, self.c_ap, self.n, self.c_xp, self.c_yp, self.c_wp,
                              0)

    def cpu_flops(self):
        return float(self.cs) * 2 * self.d * self.n ** (self.d + 1)


class BatchedSquare(Workload):
    """kronmult{d}_batched (distinct outputs), FP64 / FP32 / split."""

    def __init__(self, d=6, n=4, batch=512, precision="f64", dist="uniform", seed=SEED,
                 sweep=False):
        rng = np.random.default_rng(seed)
        self.d, self.n, self.batch, self.precision = d, n, batch, precision
        self.dist, self.seed, self.sweep = dist, seed, sweep
        self.L = n ** d
        if dist == "uniform":
            self.A = rng.uniform(-1, 1, n * n * d * batch)
        else:
            self.A = rng.standard_normal(n * n * d * batch) / np.sqrt(n)
        self.X = rng.uniform(-1, 1, self.L * batch)
        self.dtype = {"f64": "f64", "f32": "f32", "split": "f64 storage, hi+lo f32 math"}[
            precision]
        self.name = f"kronmult{d}_batched n={n} batch={batch} {precision}"

    def esize(self):
        return 4 if self.precision == "f32" else 8

    def flops(self):
        return float(self.batch) * 2 * self.d * self.n ** (self.d + 1)

    def alg_bytes(self):
        return self.esize() * float(self.batch) * (3 * self.L + self.d * self.n * self.n)

    def setup(self, torch, kb, mode, e2e=True):
        dev = torch.device("cuda")
        dt = torch.float32 if self.precision == "f32" else torch.float64
        self.kb = kb
        self.dA = torch.from_numpy(self.A).to(dev, dt)
        self.dX = torch.from_numpy(self.X).to(dev, dt)
        self.dY = torch.zeros(self.L * self.batch, dtype=dt, device=dev)
        # the caller-owned W of the reference's contract, as large as the
        # library's query asks
        need = kb.lib().kron_batched_workspace_bytes(self.d, self.n, self.batch)
        self.dW = torch.empty(max(1, need // 8), dtype=dt, device=dev) if need else None
        # vectors beyond shared memory: one slab-cluster launch for d=6 n=6
        # (FP64, FP32), one cluster two-phase launch for d=6 n=7..8 (FP64),
        # n=7..8 (FP32) and d=5 n=8 (FP64), else the two-phase path's two
        # launches
        d, n, prec = self.d, self.n, self.precision
        if not need:
            self.launches_per_step = 1
        elif d == 6 and n == 6 and prec == "f64" and self.batch >= 512:
            # the slab-cluster kernel and, concurrently on a second stream,
            # the cluster two-phase kernel on the SMs the slab clusters leave
            # idle (a share of the entries)
            self.launches_per_step = 2
        elif d == 6 and n == 6 and prec in ("f64", "f32"):
            self.launches_per_step = 1
        else:
            fp64 = prec == "f64"
            cluster = (d == 6 and (6 if fp64 else 7) <= n <= 8 and prec != "split") or \
                (fp64 and d == 5 and n == 8)
            self.launches_per_step = 1 if cluster else 2
        self.e2e_pipeline = (f"{min(E2E_CHUNKS, self.batch)} chunks of entries; uploads, calls "
                             "and downloads overlapped on 3 streams")
        if not e2e:
            return
        self.h = {k: v.cpu().pin_memory() for k, v in dict(A=self.dA, X=self.dX,
                                                          Y=self.dY).items()}
        self.hYout = torch.empty_like(self.h["Y"]).pin_memory()
        self.h2d_bytes = sum(v.numel() * v.element_size() for v in self.h.values())
        self.d2h_bytes = self.hYout.numel() * self.hYout.element_size()

    def release(self, torch):
        for k in ("dA", "dX", "dY", "dW", "h", "hYout"):
            if hasattr(self, k):
                delattr(self, k)
        torch.cuda.empty_cache()

    def comparison(self, torch, timeit):
        """The precision sweep (the headline's config): FP64, FP32 and split
        (hi+lo FP32 arithmetic on FP64 data) at n = 4 and n = 6 on this
        batch, each timed like the headline (mean of 3 steps, L2 flushed
        between) and checked against the reference's FP64 output of the same
        inputs; the headline's own case is timed again here for the speed-up
        ratios."""
        if not self.sweep:
            return None
        peaks, _ = read_peaks()
        out = {}
        for n in (4, 6):
            yref = None
            ms = {}
            for prec in ("f64", "f32", "split"):
                own = (n == self.n and prec == self.precision)
                w = self if own else BatchedSquare(self.d, n, self.batch, prec, self.dist,
                                                   self.seed)
                if not own:
                    w.setup(torch, self.kb, "atomic", e2e=False)
                if yref is None:
                    yref = w.reference_y()
                t = timeit(w.step)
                err = w.check(torch, yref)
                gbs = w.alg_bytes() / t / 1e6
                ms[prec] = t
                out[f"n{n}_{prec}"] = {
                    "ms_per_step": round(t, 4), "value": round(w.flops() / t / 1e6, 2),
                    "unit": "GFLOP/s", "hbm_gbs": round(gbs, 1),
                    "hbm_frac": round(gbs / peaks["hbm_gbs"], 4),
                    "max_rel_err_vs_fp64_reference": err["max_rel_err"],
                    "max_abs_err_vs_fp64_reference": err["max_abs_err"],
                    "launches_per_step": w.launches_per_step}
                if n == 4 and prec == "f64":
                    out["n4_repeated_apply"] = self._repeated_apply(torch, w)
                if not own:
                    w.release(torch)
                    del w
            out[f"n{n}_speedup_f32_over_f64"] = round(ms["f64"] / ms["f32"], 3)
            out[f"n{n}_speedup_split_over_f64"] = round(ms["f64"] / ms["split"], 3)
        out["reference_output"] = ("oracle/_ref (the reference's OpenMP build, recursive "
                                   "variant) on the same inputs, whole batch, FP64")
        return out

    def _repeated_apply(self, torch, w, reps=50):
        """A solver's repeated apply: the same factors A applied `reps` times
        back to back (no L2 flush between), without and then with A kept in
        L2 by kron_l2_persist_async; mean microseconds per apply."""
        kb = self.kb
        res = {}
        for persist in (False, True):
            if persist:
                kb.l2_persist(w.dA)
            try:
                w.step()
                torch.cuda.synchronize()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(reps):
                    w.step()
                b.record()
                torch.cuda.synchronize()
                res["us_per_apply_l2_persist" if persist else "us_per_apply"] = round(
                    1e3 * a.elapsed_time(b) / reps, 2)
            finally:
                if persist:
                    kb.l2_persist_reset()
        res["a_bytes"] = int(w.dA.numel() * w.dA.element_size())
        res["apply_bytes"] = w.alg_bytes()
        res["note"] = (f"{reps} applies of the same A back to back; the window keeps A "
                       "(the fixed operand) in L2 while X and Y stream")
        return res

    def step(self):
        kb = self.kb
        if self.precision == "f32":
            kb.kronmult_batched_f32(self.d, self.n, self.dA, self.dX, self.dY, self.dW)
        elif self.precision == "split":
            kb.kronmult_batched_split(self.d, self.n, self.dA, self.dX, self.dY, self.dW)
        else:
            kb.kronmult_batched(self.d, self.n, self.dA, self.dX, self.dY, self.dW)

    def e2e_step(self):
        # per chunk of entries: A, X and Y columns up, the library call, Y
        # columns down (same bytes as one call, overlapped on 3 streams)
        import torch

        kb, d, n, L, h = self.kb, self.d, self.n, self.L, self.h
        f = {"f32": kb.kronmult_batched_f32, "split": kb.kronmult_batched_split}.get(
            self.precision, kb.kronmult_batched)
        nc = min(E2E_CHUNKS, self.batch)
        chunks = []
        for c in range(nc):
            b0, b1 = c * self.batch // nc, (c + 1) * self.batch // nc
            a0, a1 = b0 * d * n * n, b1 * d * n * n
            x0, x1 = b0 * L, b1 * L
            W = self.dW[x0:x1] if self.dW is not None else None
            h2d = [(self.dA[a0:a1], h["A"][a0:a1]), (self.dX[x0:x1], h["X"][x0:x1]),
                   (self.dY[x0:x1], h["Y"][x0:x1])]

            def run(s, a0=a0, a1=a1, x0=x0, x1=x1, W=W):
                f(d, n, self.dA[a0:a1], self.dX[x0:x1], self.dY[x0:x1], W, stream=s)

            chunks.append((h2d, run, [(self.hYout[x0:x1], self.dY[x0:x1])]))
        self.run_pipeline(torch, [], chunks)

    def cpu_setup(self, sample_entries):
        self.cs = min(self.batch, sample_entries)
        self.cA = self.A[: self.cs * self.d * self.n * self.n].copy()
        self.cX = self.X[: self.cs * self.L].copy()
        self.cY = np.zeros(self.cs * self.L)
        self.cW = np.zeros(self.cs * self.L)
        return self.cs

    def cpu_step(self, ref):
        Xc = self.cX.copy()  # the reference clobbers X
        ref.kronmult_batched(self.d, self.n, self.cA, Xc, self.cY, self.cW)

    def cpu_flops(self):
        return float(self.cs) * 2 * self.d * self.n ** (self.d + 1)


class UnevenBatch(Workload):
    """20000 entries, d ~ U{1..6}, every m_l, n_l ~ U{2,3,4,6,8}: one plan
    (kron_vplan), persistent launches, replayed as a CUDA graph."""

    def __init__(self, nent=20000, seed=SEED + 4):
        rng = np.random.default_rng(seed)
        sizes = np.array([2, 3, 4, 6, 8])
        self.shapes = np.zeros((nent, 13), dtype=np.int32)
        a_off, x_off, y_off = [], [], []
        na = nx = ny = 0
        self.flop = 0.0
        import oracle as _o  # flop counts only (host arithmetic)
        for k in range(nent):
            d = int(rng.integers(1, 7))
            m = rng.choice(sizes, size=d)
            n = rng.choice(sizes, size=d)
            self.shapes[k, 0] = d
            self.shapes[k, 1:1 + 2 * d:2] = m
            self.shapes[k, 2:2 + 2 * d:2] = n
            for l in range(6):
                a_off.append(na)
                if l < d:
                    na += int(m[l] * n[l])
            x_off.append(nx)
            nx += int(np.prod(n))
            y_off.append(ny)
            ny += int(np.prod(m))
            self.flop += min(_o.flops_forward(m, n), _o.flops_backward(m, n))
        self.A = rng.uniform(-1, 1, na)
        self.X = rng.uniform(-1, 1, nx)
        self.ny = ny
        self.a_off, self.x_off, self.y_off = (np.array(v, dtype=np.int64) for v in
                                              (a_off, x_off, y_off))
        self.batch = nent
        self.name = (f"uneven batch: {nent} entries, d~U(1..6), m,n~U{{2,3,4,6,8}}, "
                     f"one vplan (persistent launches)")

    def flops(self):
        return self.flop

    def alg_bytes(self):
        return 8.0 * (self.X.size + 2 * self.ny + self.A.size)

    def setup(self, torch, kb, mode):
        dev = torch.device("cuda")
        self.kb = kb
        self.plan = kb.VPlan(self.shapes)
        self.dA = torch.from_numpy(self.A).to(dev)
        self.dX = torch.from_numpy(self.X).to(dev)
        self.dY = torch.zeros(self.ny, dtype=torch.float64, device=dev)
        self.pA = (self.dA.data_ptr() + 8 * torch.from_numpy(self.a_off)).to(dev)
        self.pX = (self.dX.data_ptr() + 8 * torch.from_numpy(self.x_off)).to(dev)
        self.pY = (self.dY.data_ptr() + 8 * torch.from_numpy(self.y_off)).to(dev)
        wb = self.plan.workspace_bytes
        self.dW = torch.empty(max(1, wb // 8), dtype=torch.float64, device=dev) if wb else None
        self.h = {k: v.cpu().pin_memory() for k, v in dict(A=self.dA, X=self.dX, Y=self.dY,
                                                          pA=self.pA, pX=self.pX,
                                                          pY=self.pY).items()}
        self.hYout = torch.empty_like(self.h["Y"]).pin_memory()
        self.h2d_bytes = sum(v.numel() * v.element_size() for v in self.h.values())
        self.d2h_bytes = self.hYout.numel() * 8
        self.launches_per_step = 1  # one persistent kernel (after a counter memset)

    def step(self):
        self.plan.execute(self.pA, self.pX, self.pY, self.dW)

    def comparison(self, torch, timeit):
        """The same entries as one plain kronmult{d}_vbatched call per
        (d, shape) group, captured as one CUDA graph (and as host launches),
        against the plan's persistent launches."""
        import ctypes as C

        kb = self.kb
        lib = kb.lib()
        dev = self.dA.device
        self.dY.zero_()
        self.step()
        y_plan = self.dY.clone()
        groups = {}
        for k in range(self.batch):
            d = int(self.shapes[k, 0])
            groups.setdefault(tuple(int(v) for v in self.shapes[k, :1 + 2 * d]), []).append(k)
        pa, px, py, glist = [], [], [], []
        wmax = 0
        for key, ks in sorted(groups.items()):
            d = key[0]
            m = (C.c_int * d)(*key[1::2])
            n = (C.c_int * d)(*key[2::2])
            wmax = max(wmax, lib.kron_vbatched_workspace_bytes(d, m, n, len(ks)))
            glist.append((d, list(key[1:]), len(pa), len(px), len(ks)))
            for k in ks:
                pa.extend(int(self.a_off[6 * k + l]) for l in range(d))
                px.append(int(self.x_off[k]))
                py.append(int(self.y_off[k]))
        gA = (self.dA.data_ptr() + 8 * torch.tensor(pa, dtype=torch.int64)).to(dev)
        gX = (self.dX.data_ptr() + 8 * torch.tensor(px, dtype=torch.int64)).to(dev)
        gY = (self.dY.data_ptr() + 8 * torch.tensor(py, dtype=torch.int64)).to(dev)
        gW = torch.empty(max(1, wmax // 8), dtype=torch.float64, device=dev)
        fns = {d: getattr(lib, f"kronmult{d}_vbatched_async") for d in range(1, 7)}

        def run_groups():
            st = torch.cuda.current_stream().cuda_stream
            for d, mn, ia, ix, cnt in glist:
                rc = fns[d](*mn, gA.data_ptr() + 8 * ia, gX.data_ptr() + 8 * ix,
                            gY.data_ptr() + 8 * ix, gW.data_ptr(), wmax, cnt, st)
                if rc != 0:
                    raise RuntimeError(f"kronmult{d}_vbatched_async failed: {rc}")

        ms_host = timeit(run_groups, reps=2)
        graph = torch.cuda.CUDAGraph()
        cs = torch.cuda.Stream()
        cs.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(cs):
            with torch.cuda.graph(graph, stream=cs):
                run_groups()
        torch.cuda.current_stream().wait_stream(cs)
        ms_graph = timeit(graph.replay)
        self.dY.zero_()
        graph.replay()
        torch.cuda.synchronize()
        err = max_rel_err(torch, self.dY, y_plan)
        del graph
        flop = self.flops()
        return {"per_group_calls": {
            "groups": len(glist), "ms_per_step_graph": round(ms_graph, 4),
            "value_graph": round(flop / ms_graph / 1e6, 2),
            "ms_per_step_host_launches": round(ms_host, 4),
            "value_host_launches": round(flop / ms_host / 1e6, 2), "unit": "GFLOP/s",
            "max_rel_err_vs_plan": err,
            "launch": "one kronmult{d}_vbatched call per (d, shape) group"}}

    def e2e_step(self):
        for k in ("A", "X", "Y", "pA", "pX", "pY"):
            getattr(self, "d" + k if k in ("A", "X", "Y") else k).copy_(self.h[k],
                                                                       non_blocking=True)
        self.step()
        self.hYout.copy_(self.dY, non_blocking=True)

    def cpu_setup(self, sample_entries):
        self.cs = min(self.batch, sample_entries)
        self.cY = np.zeros(self.ny)
        A, X, Y = self.A, self.X, self.cY
        self.c_ap = (A.ctypes.data + 8 * self.a_off[: 6 * self.cs]).astype(np.uint64)
        self.c_xp = (X.ctypes.data + 8 * self.x_off[: self.cs]).astype(np.uint64)
        self.c_yp = (Y.ctypes.data + 8 * self.y_off[: self.cs]).astype(np.uint64)
        return self.cs

    def cpu_step(self, ref):
        # the reference's kronmult{d}_vbatched, one entry per call, entries over
        # OpenMP threads (recursive variant: its Alg. 993 workspace sizing is
        # wrong for rectangular A)
        ref.kronmult_vbatched_entries(self.shapes[: self.cs], self.c_ap, self.c_xp, self.c_yp)

    def cpu_flops(self):
        import oracle as _o
        tot = 0.0
        for k in range(self.cs):
            d = int(self.shapes[k, 0])
            m = self.shapes[k, 1:1 + 2 * d:2]
            n = self.shapes[k, 2:2 + 2 * d:2]
            tot += min(_o.flops_forward(m, n), _o.flops_backward(m, n))
        return tot


class XbatchedBig(Workload):
    """d=6, n=8 (262144-element vectors), 1024 entries, outputs drawn with
    replacement from 716 (aliasing), every A_l from a pool of 32 random 8x8
    matrices per dimension, N(0,1)/sqrt(8); xbatched layout, atomic mode."""

    def __init__(self, batch=1024, nout=716, d=6, n=8, npool=32, seed=SEED + 5):
        rng = np.random.default_rng(seed)
        self.d, self.n, self.batch, self.npool, self.nout = d, n, batch, npool, nout
        self.L = n ** d
        self.Apool = rng.standard_normal(n * n * npool * d) / np.sqrt(n)
        self.aidx = rng.integers(0, npool, size=(batch, d))
        self.ylist = rng.integers(0, nout, size=batch)
        self.ndistinct = len(set(self.ylist.tolist()))
        self.xseed = seed + 1
        self.name = (f"kronmult6_xbatched n=8 FP64, {batch} entries, outputs drawn from {nout} "
                     f"({self.ndistinct} distinct), A pool {npool}/dim")

    def flops(self):
        return float(self.batch) * 2 * self.d * self.n ** (self.d + 1)

    def alg_bytes(self):
        return 8.0 * (self.L * self.batch + 2 * self.L * self.ndistinct + self.Apool.size)

    def a_offsets(self):
        l = np.arange(self.d)[None, :]
        return (self.n * self.n * (l * self.npool + self.aidx)).reshape(-1)

    def setup(self, torch, kb, mode):
        dev = torch.device("cuda")
        self.kb = kb
        g = torch.Generator(device=dev)
        g.manual_seed(self.xseed)
        self.dA = torch.from_numpy(self.Apool).to(dev)
        self.dX = torch.rand(self.L * self.batch, dtype=torch.float64, device=dev,
                             generator=g) * 2 - 1
        self.dY = torch.zeros(self.L * self.nout, dtype=torch.float64, device=dev)
        self.nw = 128
        self.dW = torch.empty(self.L * self.nw, dtype=torch.float64, device=dev)
        self.pA = (self.dA.data_ptr() + 8 * torch.from_numpy(self.a_offsets())).to(dev)
        self.pX = (self.dX.data_ptr() + 8 * self.L * torch.arange(self.batch)).to(dev)
        self.pY = (self.dY.data_ptr() + 8 * self.L * torch.from_numpy(self.ylist)).to(dev)
        self.pW = (self.dW.data_ptr() + 8 * self.L * torch.arange(self.nw)).to(dev)
        self.launches_per_step = 1
        # e2e host copies: X, Y, A pool and the pointer arrays
        self.h = {k: v.cpu().pin_memory() for k, v in dict(A=self.dA, X=self.dX, Y=self.dY,
                                                          pA=self.pA, pX=self.pX,
                                                          pY=self.pY).items()}
        self.hYout = torch.empty_like(self.h["Y"]).pin_memory()
        self.h2d_bytes = sum(v.numel() * v.element_size() for v in self.h.values())
        self.d2h_bytes = self.hYout.numel() * 8

    def step(self):
        self.kb.kronmult_xbatched(self.d, self.n, self.pA, self.n, self.pX, self.pY, self.pW,
                                  subbatch=self.nw // 2)

    def comparison(self, torch, timeit):
        """The same xbatched call with the cluster kernel on CUDA-core FMAs
        instead of the FP64 tensor cores (through the tuning table), and the
        split hi+lo FP32 path against the FP64 path on the batched layout of
        the same entries (split has no aliasing-output form)."""
        kb, d, n, L, B = self.kb, self.d, self.n, self.L, self.batch
        flop = self.flops()
        out = {}
        self.dY.zero_()
        self.step()
        y_tc = self.dY.clone()
        kb.tune_set(d, n, "f64", "big", 2 | kb.BIG_CUDA_CORES)
        try:
            ms = timeit(self.step)
            self.dY.zero_()
            self.step()
            torch.cuda.synchronize()
            out["fp64_cuda_cores"] = {
                "ms_per_step": round(ms, 4), "value": round(flop / ms / 1e6, 2),
                "unit": "GFLOP/s", "max_rel_err_vs_fp64_tensor": max_rel_err(torch, self.dY, y_tc),
                "kernel": "kron_big_kernel, 8x8 mode products as DFMA (no mma.sync)"}
        finally:
            kb.tune_set(d, n, "f64", None)
        # batched layout: entry k's factors gathered from the pool, X as is,
        # one output column per entry
        aoff = torch.from_numpy(self.a_offsets()).to(self.dA.device)
        Ab = (self.dA[aoff[:, None] + torch.arange(n * n, device=self.dA.device)]).reshape(-1)
        Yb = torch.zeros(L * B, dtype=torch.float64, device=self.dA.device)
        Wb = torch.empty(L * B, dtype=torch.float64, device=self.dA.device)
        ms64 = timeit(lambda: kb.kronmult_batched(d, n, Ab, self.dX, Yb, Wb))
        Yb.zero_()
        kb.kronmult_batched(d, n, Ab, self.dX, Yb, Wb)
        y64 = Yb.clone()
        # split on the CUDA cores (two-phase launches), forced through the
        # tuning table: the built-in choice at d = 6, n = 8 is the
        # tensor-core form below
        kb.tune_set(d, n, "split", "large")
        try:
            ms_sp = timeit(lambda: kb.kronmult_batched_split(d, n, Ab, self.dX, Yb, Wb))
            Yb.zero_()
            kb.kronmult_batched_split(d, n, Ab, self.dX, Yb, Wb)
            torch.cuda.synchronize()
        finally:
            kb.tune_set(d, n, "split", None)
        out["batched_fp64"] = {"ms_per_step": round(ms64, 4),
                               "value": round(flop / ms64 / 1e6, 2), "unit": "GFLOP/s",
                               "layout": f"batched, the same {B} entries, distinct outputs"}
        out["batched_split"] = {
            "ms_per_step": round(ms_sp, 4), "value": round(flop / ms_sp / 1e6, 2),
            "unit": "GFLOP/s", "max_rel_err_vs_fp64": max_rel_err(torch, Yb, y64),
            "arithmetic": "hi+lo FP32 parts of A and X, three cross products with compensated "
                          "FP32 sums, CUDA cores"}
        # the same split call with the 8x8 mode products as exact BF16 slice
        # products on the tcgen05 tensor cores (the built-in choice)
        kb.tune_set(d, n, "split", "split_tc")
        try:
            ms_tc = timeit(lambda: kb.kronmult_batched_split(d, n, Ab, self.dX, Yb, Wb))
            Yb.zero_()
            kb.kronmult_batched_split(d, n, Ab, self.dX, Yb, Wb)
            torch.cuda.synchronize()
            out["batched_split_tc"] = {
                "ms_per_step": round(ms_tc, 4), "value": round(flop / ms_tc / 1e6, 2),
                "unit": "GFLOP/s", "max_rel_err_vs_fp64": max_rel_err(torch, Yb, y64),
                "arithmetic": "six 8-bit slices of A and X per mode product, BF16 tcgen05.mma "
                              "with FP32 accumulators (exact), FP64 reconstruction"}
        finally:
            kb.tune_set(d, n, "split", None)
        del Ab, Yb, Wb, y_tc
        torch.cuda.empty_cache()
        return out

    def reference_y(self):
        """The reference's kronmult6_xbatched over the whole batch on the
        device's X (generated on the GPU), Y from zero; cached."""
        if self._yref is None:
            import oracle

            ref = oracle.Reference("recur")
            L, B = self.L, self.batch
            X = self.dX.cpu().numpy()
            Y = np.zeros(L * self.nout)
            W = np.zeros(L * B)
            ap = (self.Apool.ctypes.data + 8 * self.a_offsets()).astype(np.uint64)
            xp = (X.ctypes.data + 8 * L * np.arange(B)).astype(np.uint64)
            yp = (Y.ctypes.data + 8 * L * self.ylist).astype(np.uint64)
            wp = (W.ctypes.data + 8 * L * np.arange(B)).astype(np.uint64)
            ref.kronmult_xbatched(self.d, self.n, ap, self.n, xp, yp, wp, 0)
            del W, X
            self._yref = Y
        return self._yref

    def e2e_step(self):
        self.dA.copy_(self.h["A"], non_blocking=True)
        self.dX.copy_(self.h["X"], non_blocking=True)
        self.dY.copy_(self.h["Y"], non_blocking=True)
        self.pA.copy_(self.h["pA"], non_blocking=True)
        self.pX.copy_(self.h["pX"], non_blocking=True)
        self.pY.copy_(self.h["pY"], non_blocking=True)
        self.step()
        self.hYout.copy_(self.dY, non_blocking=True)

    def cpu_setup(self, sample_entries):
        self.cs = min(self.batch, sample_entries, 16)
        rng = np.random.default_rng(self.xseed)
        self.cX = rng.uniform(-1, 1, self.L * self.cs)
        self.cY = np.zeros(self.L * self.nout)
        self.cW = np.zeros(self.L * self.cs)
        self.c_ap = (self.Apool.ctypes.data + 8 * self.a_offsets()[: self.cs * self.d]).astype(
            np.uint64)
        self.c_xp = (self.cX.ctypes.data + 8 * self.L * np.arange(self.cs)).astype(np.uint64)
        self.c_yp = (self.cY.ctypes.data + 8 * self.L * self.ylist[: self.cs]).astype(np.uint64)
        self.c_wp = (self.cW.ctypes.data + 8 * self.L * np.arange(self.cs)).astype(np.uint64)
        return self.cs

    def cpu_step(self, ref):
        ref.kronmult_xbatched(self.d, self.n, self.c_ap, self.n, self.c_xp, self.c_yp, self.c_wp,
                              0)

    def cpu_flops(self):
        return float(self.cs) * 2 * self.d * self.n ** (self.d + 1)


class KgemmBatched(Workload):
    """kgemm_nn_batched, the reference's batched small GEMM: mm = nn = kk =
    64 (the largest size its tests sweep, test_kgemm_nn_batched.cpp:491-533),
    C_k += A_k B_k (alpha = 1, beta = 1: the accumulate form the Kronecker
    kernels call), distinct C_k, A/B/C ~ U(-1,1)."""

    def __init__(self, batch=32768, mm=64, nn=64, kk=64, seed=SEED + 6):
        rng = np.random.default_rng(seed)
        self.batch, self.mm, self.nn, self.kk = batch, mm, nn, kk
        self.A = rng.uniform(-1, 1, mm * kk * batch)
        self.B = rng.uniform(-1, 1, kk * nn * batch)
        self.C0 = rng.uniform(-1, 1, mm * nn * batch)
        self.name = f"kgemm_nn_batched {mm}x{nn}x{kk}, batch {batch}, alpha=1 beta=1, FP64"

    def flops(self):
        return 2.0 * self.mm * self.nn * self.kk * self.batch

    def alg_bytes(self):
        return 8.0 * self.batch * (self.mm * self.kk + self.kk * self.nn + 2 * self.mm * self.nn)

    def _ptrs(self, torch, base, stride):
        return (base.data_ptr() + 8 * stride * torch.arange(self.batch, dtype=torch.int64)).to(
            base.device)

    def setup(self, torch, kb, mode):
        dev = torch.device("cuda")
        self.kb = kb
        self.dA = torch.from_numpy(self.A).to(dev)
        self.dB = torch.from_numpy(self.B).to(dev)
        self.dY = torch.from_numpy(self.C0).to(dev)
        mm, nn, kk = self.mm, self.nn, self.kk
        self.pA = self._ptrs(torch, self.dA, mm * kk)
        self.pB = self._ptrs(torch, self.dB, kk * nn)
        self.pC = self._ptrs(torch, self.dY, mm * nn)
        self.ldA = torch.full((self.batch,), mm, dtype=torch.int32, device=dev)
        self.ldB = torch.full((self.batch,), kk, dtype=torch.int32, device=dev)
        self.ldC = torch.full((self.batch,), mm, dtype=torch.int32, device=dev)
        self.h = {k: v.cpu().pin_memory() for k, v in dict(A=self.dA, B=self.dB,
                                                          C=self.dY).items()}
        self.hYout = torch.empty_like(self.h["C"]).pin_memory()
        self.h2d_bytes = sum(v.numel() * v.element_size() for v in self.h.values())
        self.d2h_bytes = self.hYout.numel() * 8

    def step(self):
        self.kb.kgemm_batched("nn", self.mm, self.nn, self.kk, 1.0, self.pA, self.ldA, self.pB,
                              self.ldB, 1.0, self.pC, self.ldC)

    def comparison(self, torch, timeit):
        """The same call on the CUDA-core tile kernel (64x64 tiles, FMA) that
        larger entries use, against the tensor-core kernel of the headline."""
        self.dY.zero_()
        self.step()
        y_tc = self.dY.clone()
        os.environ["KRON_KGEMM_CUDA_CORES"] = "1"
        try:
            ms = timeit(self.step)
            self.dY.zero_()
            self.step()
            torch.cuda.synchronize()
            err = max_rel_err(torch, self.dY, y_tc)
        finally:
            del os.environ["KRON_KGEMM_CUDA_CORES"]
        return {"cuda_cores": {"ms_per_step": round(ms, 4),
                               "value": round(self.flops() / ms / 1e6, 2), "unit": "GFLOP/s",
                               "max_rel_err_vs_tensor_cores": err,
                               "kernel": "64x64 tiles, K by 16, CUDA-core FMA"}}

    def e2e_step(self):
        self.dA.copy_(self.h["A"], non_blocking=True)
        self.dB.copy_(self.h["B"], non_blocking=True)
        self.dY.copy_(self.h["C"], non_blocking=True)
        self.step()
        self.hYout.copy_(self.dY, non_blocking=True)

    def cpu_setup(self, sample_entries):
        self.cs = min(self.batch, sample_entries)
        mm, nn, kk, cs = self.mm, self.nn, self.kk, self.cs
        self.cY = np.zeros(mm * nn * cs)
        self.c_ap = (self.A.ctypes.data + 8 * mm * kk * np.arange(cs)).astype(np.uint64)
        self.c_bp = (self.B.ctypes.data + 8 * kk * nn * np.arange(cs)).astype(np.uint64)
        self.c_cp = (self.cY.ctypes.data + 8 * mm * nn * np.arange(cs)).astype(np.uint64)
        self.c_ld = [np.full(cs, v, dtype=np.int32) for v in (mm, kk, mm)]
        return cs

    def cpu_step(self, ref):
        ref.kgemm_batched("nn", self.mm, self.nn, self.kk, 1.0, self.c_ap, self.c_ld[0],
                          self.c_bp, self.c_ld[1], 1.0, self.c_cp, self.c_ld[2])

    def cpu_flops(self):
        return 2.0 * self.mm * self.nn * self.kk * self.cs


def make_workload(cfg, precision, entries=0, n=6):
    """The workload of --config cfg (n: config 3's size); entries > 0 scales
    its batch down (or up) for small profiling cases (configs 1, 3, 4, 5
    and 6; outputs of config 5 keep their 716:1024 ratio)."""
    if cfg == 1:
        return BatchedSquare(6, 4, entries or 512, "f64", "uniform")
    if cfg == 2:
        return XbatchedOverlap()
    if cfg == 3:
        return BatchedSquare(6, n, entries or 4096, precision, "normal", sweep=not entries)
    if cfg == 4:
        return UnevenBatch(nent=entries or 20000)
    if cfg == 5:
        if entries:
            return XbatchedBig(batch=entries, nout=max(1, entries * 716 // 1024))
        return XbatchedBig()
    if cfg == 6:
        return KgemmBatched(batch=entries or 32768)
    raise SystemExit(f"--config {cfg} not available in this bench")


# ---------------------------------------------------------------- helpers
def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_key(args):
    """Key of a workload in the committed ncu summaries: `cfgN` for FP64,
    atomic mode and the full batch (config 3 at n = 4), with `-f32`, `-split`,
    `-segmented`, `-n6`, `-eK` appended for the variants."""
    key = f"cfg{args.config}"
    if args.precision != "f64":
        key += f"-{args.precision}"
    if args.mode != "atomic":
        key += f"-{args.mode}"
    if args.config == 3 and getattr(args, "n", 4) != 4:
        key += f"-n{args.n}"
    if getattr(args, "entries", 0):
        key += f"-e{args.entries}"
    return key


def read_profile_traffic(key):
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu
    summary (profiles/*.md line `traffic_bytes_per_launch[<key>]: <bytes>`)."""
    import glob
    import re

    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(p) as f:
            for line in f:
                m = re.match(rf"\s*traffic_bytes_per_launch\[{re.escape(key)}\]:\s*([0-9.eE+]+)",
                             line)
                if m:
                    return float(m.group(1)), os.path.relpath(p, ROOT)
    return None, None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.dev = device_index
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def max_over_ranks(dist, values, device):
    """Element-wise max of `values` over all ranks (the slowest replica sets
    every time); the values unchanged without a process group."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------- reference arm
def run_reference(args, world, rank):
    """The reference's own CPU (OpenMP) implementation of the same workload,
    on the host cores: oracle/_ref, compiled from the reference sources by
    oracle/Makefile.  Without that build it prints the `unavailable` line."""
    if rank != 0:
        return
    import oracle

    wl = make_workload(args.config, args.precision, args.entries, args.n)
    if oracle.Reference.available("recur"):
        ref = oracle.Reference("recur")
        kind = "reference"
        cores = ref.max_threads()
    else:
        raise SystemExit(json.dumps({"impl": "reference",
                                     "unavailable": "oracle/_ref not built on this machine"}))
    sample = wl.cpu_setup(args.cpu_sample)
    for _ in range(args.warmup):
        wl.cpu_step(ref)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        wl.cpu_step(ref)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = wl.cpu_flops() * len(times) / tot / 1e9
    line = {"metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s",
            "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * tot / len(times), 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "sample_entries": sample},
            "cpu_baseline": {"value": round(value, 3), "unit": "GFLOP/s", "cores": cores,
                             "kind": kind,
                             "sample": f"{sample} of {wl.batch} entries per step, "
                                       f"OpenMP {cores} threads, recursive variant"},
            "e2e": {"value": round(value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(args, world, rank, local):
    import torch

    import kronmult_b200 as kb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    kb.lib()
    wl = make_workload(args.config, args.precision, args.entries, args.n)
    tuned = None
    if args.variant and hasattr(wl, "n") and hasattr(wl, "d"):
        # force one kernel form for this square (d, n, precision)
        name, _, q = args.variant.partition(":")
        kb.tune_set(wl.d, wl.n, getattr(wl, "precision", "f64"), name, int(q or 0))
        tuned = f"{name}:{int(q or 0)} (forced)"
    elif args.autotune and hasattr(wl, "n") and hasattr(wl, "d"):
        # pick the kernel variant for this square (d, n, precision) before
        # anything is timed
        prec = getattr(wl, "precision", "f64")
        v, q, us = kb.autotune(wl.d, wl.n, prec, batch=min(wl.batch, 4096))
        tuned = f"{v}:{q} ({us:.1f} us on the synthetic batch)"
    wl.setup(torch, kb, args.mode)
    flush_w = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    flush_r = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sink = torch.empty(1, dtype=torch.float32, device="cuda")

    class _Flush:
        """L2 flush between timed steps: write 256 MB (evicts everything),
        then read another 256 MB so the L2 holds clean lines only and the
        next step does not pay for the flush's own write-backs."""

        @staticmethod
        def zero_():
            flush_w.zero_()
            torch.sum(flush_r, dim=0, out=sink[0])

    flush = _Flush()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        wl.step()
        flush.zero_()
    barrier()
    step = wl.step
    graph = None
    if not args.no_graph:
        # one library call captured once and replayed: the device-timed steps
        # then carry no host launch latency
        graph = torch.cuda.CUDAGraph()
        cs = torch.cuda.Stream()
        cs.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(cs):
            with torch.cuda.graph(graph, stream=cs):
                wl.step()
        torch.cuda.current_stream().wait_stream(cs)
        torch.cuda.synchronize()
        step = graph.replay
        for _ in range(2):
            step()
            flush.zero_()
        barrier()
    clock = ClockSampler(local) if rank == 0 else None
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        starts[i].record()
        step()
        ends[i].record()
        flush.zero_()
    barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    tot_ms = sum(step_ms)

    # e2e through the public API with pinned host buffers
    for _ in range(max(1, args.warmup // 2)):
        wl.e2e_step()
    barrier()
    e_s = torch.cuda.Event(enable_timing=True)
    e_e = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 10))
    e_s.record()
    for _ in range(e2e_steps):
        wl.e2e_step()
    e_e.record()
    barrier()
    e2e_ms = e_s.elapsed_time(e_e)
    clocks = clock.stop() if clock else None

    tot_ms, e2e_ms = max_over_ranks(dist, [tot_ms, e2e_ms], "cuda")

    # the stated error (rank 0, outside the timed region): one step from
    # Y = 0 against the reference's own output on the same inputs
    err = None
    if rank == 0 and not args.no_check:
        import oracle

        if oracle.Reference.available("recur"):
            err = wl.check(torch)
            err["against"] = ("the reference's own output (oracle/_ref: its OpenMP build, "
                              "recursive variant) on the same inputs, whole batch, FP64")
        else:
            err = {"unavailable": "oracle/_ref not built on this machine"}

    # comparison legs (rank 0, N=1 only; outside the timed region): other
    # kernels on the same workload, each with its error against the FP64
    # reference output
    comparison = None
    if rank == 0 and world == 1 and not args.no_compare and hasattr(wl, "comparison"):
        def timeit(fn, reps=3):
            fn()
            flush.zero_()
            torch.cuda.synchronize()
            evs = []
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                fn()
                b.record()
                flush.zero_()
                evs.append((a, b))
            torch.cuda.synchronize()
            return sum(a.elapsed_time(b) for a, b in evs) / reps

        comparison = wl.comparison(torch, timeit)

    # CPU baseline (rank 0, N=1 only): the reference's OpenMP build, bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(wl, args)

    if rank == 0:
        peaks, peak_src = read_peaks()
        flops = wl.flops()
        sec = tot_ms / 1e3
        value = world * flops * args.steps / sec / 1e9
        gbs = wl.alg_bytes() * args.steps / sec / 1e9
        per_launch_s = sec / (args.steps * wl.launches_per_step)
        traffic, tsrc = read_profile_traffic(profile_key(args))
        if args.config == 2 or args.config == 5:
            fp64 = measure_fp64_peak(torch)
            roof = {"bound": "tensor", "achieved": round(flops / wl.launches_per_step /
                                                         per_launch_s / 1e12, 3),
                    "peak": round(fp64, 3), "unit": "TFLOP/s",
                    "frac": round(flops / wl.launches_per_step / per_launch_s / 1e12 / fp64, 4),
                    "traffic": traffic,
                    "peak_source": "FP64 tensor-core (mma.sync f64) throughput measured live "
                                   "by kron_measure_fp64_peak; MEASURED_PEAKS.json has no "
                                   "FP64 figure",
                    "hbm_gbs_achieved": round(gbs, 1),
                    "hbm_frac": round(gbs / peaks["hbm_gbs"], 4)}
        else:
            roof = {"bound": "hbm", "achieved": round(wl.alg_bytes() / wl.launches_per_step /
                                                      per_launch_s / 1e9, 1),
                    "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": round(wl.alg_bytes() / wl.launches_per_step / per_launch_s / 1e9 /
                                  peaks["hbm_gbs"], 4),
                    "traffic": traffic, "peak_source": f"MEASURED_PEAKS.json ({peak_src})"}
        if tsrc:
            roof["traffic_source"] = tsrc
        if wl.launches_per_step > 1:
            # achieved and traffic are per launch: the step's bytes over the
            # step's time (concurrent launches) or each launch's share
            roof["launches_per_step"] = wl.launches_per_step
        line = {"metric": METRIC, "value": round(value, 2), "unit": "GFLOP/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(tot_ms / args.steps, 5), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype,
                "data": "synthetic (seeded PCG64; no public dataset exists)",
                "config": {"workload": wl.name, "mode": args.mode,
                           "launch": "CUDA graph replay of one library call" if graph is not None
                           else "direct library call",
                           "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                           "l2": "flush between timed steps, outside the events: 256 MB write "
                                 "then 256 MB read (L2 left cold and clean)",
                           "alg_bytes_per_step": wl.alg_bytes(), "flops_per_step": flops,
                           "kernel_choice": tuned or "built-in order"},
                "hbm_gbs": round(world * gbs, 1),
                "roofline": roof,
                "cpu_baseline": cpu,
                "e2e": {"value": round(world * flops * e2e_steps / (e2e_ms / 1e3) / 1e9, 2),
                        "unit": "GFLOP/s", "h2d_bytes_per_step": wl.h2d_bytes,
                        "d2h_bytes_per_step": wl.d2h_bytes,
                        "ms_per_step": round(e2e_ms / e2e_steps, 4),
                        "pipeline": wl.e2e_pipeline or "one call: uploads, call, download in order"},
                "gpu_launches": args.steps * wl.launches_per_step,
                "clocks": clocks}
        if err is not None:
            line["max_rel_err"] = err.get("max_rel_err")
            line["err"] = err
        if comparison:
            line["comparison"] = comparison
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def measure_fp64_peak(torch):
    """FP64 tensor-core throughput of this GPU (mma.sync f64 chains on every
    SM, measured live by the library), TFLOP/s."""
    import kronmult_b200 as kb

    tensor, _core = kb.measure_fp64_peak()
    return tensor


def cpu_baseline(wl, args):
    import oracle

    if not oracle.Reference.available("recur"):
        return None
    ref = oracle.Reference("recur")
    sample = wl.cpu_setup(args.cpu_sample)
    wl.cpu_step(ref)
    t0 = time.perf_counter()
    n = 0
    while True:
        wl.cpu_step(ref)
        n += 1
        if time.perf_counter() - t0 > args.cpu_seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": round(wl.cpu_flops() * n / dt / 1e9, 3), "unit": "GFLOP/s",
            "cores": ref.max_threads(), "kind": "reference",
            "sample": f"{sample} of {wl.batch} entries x {n} repetitions "
                      f"({dt:.1f} s), reference OpenMP build, recursive variant"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--n", type=int, default=int(os.environ.get("KRON_BENCH_N", "6")),
                    choices=[4, 6, 8],
                    help="config 3: factor size (default 6; 8 for profiling cases with --entries)")
    ap.add_argument("--mode", default="atomic", choices=["atomic", "segmented"])
    ap.add_argument("--precision", default="f64", choices=["f64", "f32", "split"])
    ap.add_argument("--cpu-sample", type=int, default=1 << 30)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the comparison legs of configs 3, 4 and 5")
    ap.add_argument("--no-check", action="store_true",
                    help="skip the error check against the reference's output")
    ap.add_argument("--variant", default="",
                    help="force a kernel form through the tuning table: name[:param] "
                         "(mma8, pipe, sq, gen, big, large, slab, split_tc)")
    ap.add_argument("--autotune", action="store_true",
                    help="run the library's autotuner for the workload's shape first")
    ap.add_argument("--entries", type=int, default=0,
                    help="scale the batch of configs 1/3/5 (small profiling cases)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
