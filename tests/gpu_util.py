"""Helpers shared by the GPU parity tests."""
import numpy as np

CT = np.complex128


def to_dev(a):
    """Column-major (Julia layout) complex128 device buffer of a host tensor."""
    import torch
    flat = np.ascontiguousarray(np.asarray(a, dtype=CT).ravel(order="F"))
    return torch.from_numpy(flat).to("cuda")


def empty_dev(shape):
    import torch
    return torch.zeros(int(np.prod(shape)), dtype=torch.complex128, device="cuda")


def from_dev(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


def crand(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(CT)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
