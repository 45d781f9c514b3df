"""Helpers shared by the tests: numpy <-> device buffers, relative errors."""
import numpy as np


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def empty_like_dev(shape):
    import torch

    return torch.full(shape, float("nan"), dtype=torch.complex128, device="cuda")
