"""Helpers shared by the GPU parity tests."""
import numpy as np


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32).copy()).cuda()


def to_host(t, n=None):
    import torch
    torch.cuda.synchronize()
    x = t.detach().cpu().numpy().view(np.uint32)
    return x if n is None else x[:n]


def empty(n):
    import torch
    return torch.zeros(max(int(n), 1), dtype=torch.int32, device="cuda")
