"""Owner-computes sharding of a batch with overlapping outputs over several
GPUs: one process per GPU, torch.distributed (NCCL) for the exchange.

In the xbatched layout several entries may add into one output column.
kron_owner_partition (C ABI, host) gives every output index to exactly one
rank, together with every entry that writes it.  A rank builds the pointer
arrays of its own entries on its GPU from the integer lists
(kron_build_pointers_async) and runs them in one xbatched call, with atomic
adds or in the deterministic segmented mode.  Its outputs are then final:
no partial sum leaves the GPU, so the data path needs no collective.
gather() copies each rank's owned output range to every rank (one broadcast
per rank), for callers that want the whole Y everywhere; a solver that keeps
Y distributed skips it.

The reference runs one device; its aliasing contract is the one kept here
(kronmult6_pbatched.hpp:52-66, kronmult_xbatched.hpp:17-162: entries with
one Y column add up).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (Segments, _check, _torch, build_pointers, kronmult_xbatched,
               kronmult_xbatched_segmented, lib)


def owner_partition(ylist, nranks):
    """(entry_order, entry_bounds, out_bounds) of kron_owner_partition, as
    int32 numpy arrays: rank r owns outputs [out_bounds[r], out_bounds[r+1])
    and computes entries entry_order[entry_bounds[r]:entry_bounds[r+1]]."""
    y = np.ascontiguousarray(ylist, dtype=np.int32)
    order = np.empty(y.size, dtype=np.int32)
    eb = np.empty(nranks + 1, dtype=np.int32)
    ob = np.empty(nranks + 1, dtype=np.int32)
    _check(lib().kron_owner_partition(y.size, y.ctypes.data_as(C.c_void_p), nranks,
                                      order.ctypes.data_as(C.c_void_p),
                                      eb.ctypes.data_as(C.c_void_p),
                                      ob.ctypes.data_as(C.c_void_p)),
           "kron_owner_partition")
    return order, eb, ob


class OwnerShard:
    """Rank `rank`'s share of an xbatched batch given by index lists:
    entry k reads X column xlist[k] and factor blocks alist[l + k d]
    (l = 0..d-1) and adds into Y column ylist[k].

    entries      this rank's entries (increasing output, batch order within one)
    out_lo/hi    its output columns [out_lo, out_hi)
    out_bounds   every rank's output ranges (nranks + 1)
    """

    def __init__(self, d, xlist, ylist, alist, rank, nranks):
        if not 0 <= rank < nranks:
            raise ValueError(f"rank {rank} outside 0..{nranks - 1}")
        x = np.ascontiguousarray(xlist, dtype=np.int32)
        y = np.ascontiguousarray(ylist, dtype=np.int32)
        a = np.ascontiguousarray(alist, dtype=np.int32).reshape(y.size, d)
        if x.size != y.size:
            raise ValueError("xlist and ylist differ in length")
        order, eb, ob = owner_partition(y, nranks)
        self.d, self.rank, self.nranks = d, rank, nranks
        self.entries = order[eb[rank]:eb[rank + 1]]
        self.out_bounds = ob
        self.out_lo, self.out_hi = int(ob[rank]), int(ob[rank + 1])
        self.xlist = x[self.entries]
        self.ylist = y[self.entries]
        self.alist = a[self.entries].reshape(-1)
        self._dev = None   # device copies of the lists
        self._seg = None   # segmented plan, keyed by the Y pointer it was built for

    def __len__(self):
        return int(self.entries.size)

    def _lists(self):
        if self._dev is None:
            torch = _torch()
            self._dev = tuple(torch.from_numpy(v).cuda() for v in (self.alist, self.xlist,
                                                                  self.ylist))
        return self._dev

    def apply(self, n, A, astride, lda, X, xstride, Y, ystride, deterministic=False,
              stream=None):
        """Y(:, ylist[k]) += kron(A blocks of k) X(:, xlist[k]) for this rank's
        entries, on the current GPU.  A, X, Y are device float64 tensors;
        strides in elements.  deterministic: the segmented mode (bitwise
        reproducible; each output summed in batch order)."""
        if len(self) == 0:
            return
        dal, dxl, dyl = self._lists()
        pA, pX, pY = build_pointers(self.d, A, astride, dal, X, xstride, dxl, Y, ystride, dyl,
                                    stream=stream)
        if deterministic:
            key = (Y.data_ptr(), ystride)
            if self._seg is None or self._seg[0] != key:
                self._seg = (key, Segments(pY, stream=stream))
            kronmult_xbatched_segmented(self.d, n, pA, lda, pX, pY, self._seg[1], stream=stream)
        else:
            kronmult_xbatched(self.d, n, pA, lda, pX, pY, stream=stream)

    def gather(self, Y, ystride, group=None):
        """Copy every rank's owned output columns of Y (a contiguous tensor,
        column j at j * ystride) to all ranks: one broadcast per rank, from
        the owner.  Every rank of the group calls it with the same Y shape."""
        import torch.distributed as dist

        for r in range(self.nranks):
            lo, hi = int(self.out_bounds[r]) * ystride, int(self.out_bounds[r + 1]) * ystride
            hi = min(hi, Y.numel())
            if hi > lo:
                src = r if group is None else dist.get_global_rank(group, r)
                dist.broadcast(Y[lo:hi], src=src, group=group)
