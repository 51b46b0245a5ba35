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


def fidelity(sites_a, sites_b):
    """|<a|b>|^2 / (<a|a><b|b>) of two MPS given as host site lists (gauge invariant)."""
    from oracle import mps_ref as R
    ab = R.scal_prod(sites_a, sites_b)
    aa = R.scal_prod(sites_a, sites_a).real
    bb = R.scal_prod(sites_b, sites_b).real
    return abs(ab) ** 2 / (aa * bb)


class perturbed_oracle_qr:
    """Context manager: the oracle's qrq/julia_qr see inputs scaled by (1 + eps*N(0,1)) entrywise,
    the rounding-level perturbation that measures the truncated dynamics' own sensitivity."""

    def __init__(self, eps=1e-15, seed=5):
        self.eps, self.seed = eps, seed

    def __enter__(self):
        from oracle import mps_ref as R
        self.R = R
        self.orig = (R.qrq, R.julia_qr)
        rng = np.random.default_rng(self.seed)
        eps = self.eps
        oq, oj = self.orig

        def qrq(M):
            return oq(M * (1 + eps * rng.standard_normal(M.shape)))

        def jqr(M):
            return oj(M * (1 + eps * rng.standard_normal(M.shape)))
        R.qrq, R.julia_qr = qrq, jqr
        return self

    def __exit__(self, *a):
        self.R.qrq, self.R.julia_qr = self.orig
