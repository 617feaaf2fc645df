"""Helpers for the GPU tests: device copies and device pointer arrays."""
from __future__ import annotations

import numpy as np


def dev(a, dtype=None):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def ptrs(base, offsets, esize=8):
    """Device int64 tensor of addresses base + esize*offset."""
    import torch

    addr = [base.data_ptr() + esize * int(o) for o in offsets]
    return torch.tensor(addr, dtype=torch.int64, device="cuda")


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.detach().cpu().numpy()
