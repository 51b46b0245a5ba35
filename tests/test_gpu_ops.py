"""Op-level parity of the CUDA kernels with the oracle (each call goes through the C ABI)."""
import ctypes as C

import numpy as np
import pytest

from gpu_util import crand, empty_dev, from_dev, relerr, to_dev
from oracle import mps_ref as R

pytestmark = pytest.mark.gpu
TOL = 1e-12  # relative, complex128 op-level (rounding-order differences only)


def _call(ctx, name, *args):
    """Order the library stream after torch's writes and before torch's reads."""
    import torch
    from mpsb200 import _lib
    torch.cuda.synchronize()
    _lib.call(name, ctx.h, *args)
    ctx.sync()


def _p(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("m,n", [(1, 1), (2, 1), (4, 2), (8, 8), (64, 32), (100, 37), (128, 64), (512, 128), (256, 256)])
def test_qr_matches_lapack(gpu_ctx, m, n):
    rng = np.random.default_rng(m * 1000 + n)
    X = crand(rng, m, n)
    q_ref, r_ref = R.julia_qr(X)
    dX, dQ, dR = to_dev(X), empty_dev((m, n)), empty_dev((n, n))
    _call(gpu_ctx, "mpsb_op_qr", _p(dX), _p(dQ), _p(dR), m, n)
    Q, Rr = from_dev(dQ, (m, n)), from_dev(dR, (n, n))
    assert relerr(Q, q_ref) < 1e-11
    assert relerr(Rr, r_ref) < 1e-11
    assert np.abs(Q.conj().T @ Q - np.eye(n)).max() < 1e-13


def test_qr_in_place_and_rank_deficient(gpu_ctx):
    """Zero-padded product-state sites: the junk columns come from tau = 0 reflectors."""
    for (dl, d, dr) in [(1, 2, 2), (2, 2, 4), (4, 2, 8), (8, 4, 32), (16, 2, 32)]:
        site = np.zeros((dl, d, dr), dtype=np.complex128)
        site[0, :, 0] = [0.0, 1.0] + [0.0] * (d - 2)
        X = R.jr(site, dl * d, dr)
        q_ref = R.qrq(X)
        dX = to_dev(X)
        _call(gpu_ctx, "mpsb_op_qr", _p(dX), _p(dX), None, dl * d, dr)
        assert np.abs(from_dev(dX, (dl * d, dr)) - q_ref).max() < 1e-15


def test_qr_mixed_exact_zero_columns(gpu_ctx):
    rng = np.random.default_rng(7)
    X = crand(rng, 48, 24)
    X[:, 5] = 0
    X[10:, 9] = 0
    X[:, 20] = X[:, 3]          # exactly dependent column
    q_ref = R.qrq(X)
    dX, dQ = to_dev(X), empty_dev((48, 24))
    _call(gpu_ctx, "mpsb_op_qr", _p(dX), _p(dQ), None, 48, 24)
    Q = from_dev(dQ, (48, 24))
    # the span is fixed; columns after an exactly dependent one are noise-determined, so compare
    # only up to it (where the convention fixes everything) and check orthonormality overall
    assert np.abs(Q[:, :20] - q_ref[:, :20]).max() < 1e-12
    assert np.abs(Q.conj().T @ Q - np.eye(24)).max() < 1e-12


@pytest.mark.parametrize("m,n", [(64, 16), (64, 32), (200, 48), (512, 128), (1024, 300)])
def test_qr_tiny_columns_match_lapack(gpu_ctx, m, n):
    """Columns scaled down to 1e-240 (the sweeps from product states produce amplitudes of
    1e-150 and below): Householder QR is invariant under positive column scaling, Q(X D) = Q(X)
    and R(X D) = R(X) D, which LAPACK keeps through zlarfg's rescaling; so must the GPU."""
    rng = np.random.default_rng(m * 7 + n)
    X = crand(rng, m, n)
    e = rng.choice([0, 40, 80, 150, 154, 158, 162, 200, 240], size=n)
    D = 10.0 ** (-e.astype(float))
    q_ref, r_ref = R.julia_qr(X)
    dX, dQ, dR = to_dev(X * D), empty_dev((m, n)), empty_dev((n, n))
    _call(gpu_ctx, "mpsb_op_qr", _p(dX), _p(dQ), _p(dR), m, n)
    Q, Rr = from_dev(dQ, (m, n)), from_dev(dR, (n, n))
    assert np.isfinite(Q).all() and np.isfinite(Rr).all()
    assert np.abs(Q - q_ref).max() < 1e-11
    assert np.abs(Rr / D - r_ref).max() < 1e-11 * np.abs(r_ref).max()


@pytest.mark.parametrize("m,n", [(2048, 512), (1024, 300), (640, 40)])
def test_qr_blocked_path_matches_lapack(gpu_ctx, m, n):
    """Shapes beyond one cluster's shared memory (2048 x 512 is the interior site of a
    chi = 512, d = 4 chain): panel-by-panel factorisation with GEMM trailing updates."""
    rng = np.random.default_rng(m + n)
    X = crand(rng, m, n)
    q_ref, r_ref = R.julia_qr(X)
    dX, dQ, dR = to_dev(X), empty_dev((m, n)), empty_dev((n, n))
    _call(gpu_ctx, "mpsb_op_qr", _p(dX), _p(dQ), _p(dR), m, n)
    Q, Rr = from_dev(dQ, (m, n)), from_dev(dR, (n, n))
    assert relerr(Q, q_ref) < 1e-10
    assert relerr(Rr, r_ref) < 1e-10
    assert np.abs(Q.conj().T @ Q - np.eye(n)).max() < 1e-12
    assert np.abs(from_dev(dX, (m, n)) - X).max() == 0      # the input is left untouched
    dX2 = to_dev(X)                                            # in place
    _call(gpu_ctx, "mpsb_op_qr", _p(dX2), _p(dX2), None, m, n)
    assert np.abs(from_dev(dX2, (m, n)) - Q).max() < 1e-13


def test_qr_blocked_rank_deficient_padded_site(gpu_ctx):
    """A zero-padded product site at chi = 512, d = 4 (tau = 0 and junk columns) on the blocked path."""
    dl, d, dr = 512, 4, 512
    X = np.zeros((dl * d, dr), dtype=np.complex128)
    X[1, 0] = 1.0
    q_ref = R.qrq(X)
    dX = to_dev(X)
    _call(gpu_ctx, "mpsb_op_qr", _p(dX), _p(dX), None, dl * d, dr)
    Q = from_dev(dX, (dl * d, dr))
    assert np.abs(Q - q_ref).max() < 1e-12


@pytest.mark.parametrize("m,n", [(1, 1), (1, 8), (8, 1), (64, 16), (16, 64), (128, 128), (512, 131), (96, 600)])
def test_svd_matches_lapack(gpu_ctx, m, n):
    """Thin SVD (the `svd` of compressionSVD!): singular values to relative accuracy, the
    factors orthonormal and reproducing X (vectors are unique only up to phases)."""
    rng = np.random.default_rng(m * 7 + n)
    X = crand(rng, m, n)
    X[:, :: max(1, n // 5)] *= 1e-6                      # a spread of singular values
    k = min(m, n)
    s_ref = np.linalg.svd(X, compute_uv=False)
    dX, dU, dV = to_dev(X), empty_dev((m, k)), empty_dev((n, k))
    S = np.zeros(k)
    _call(gpu_ctx, "mpsb_op_svd", _p(dX), _p(dU), S.ctypes.data_as(C.POINTER(C.c_double)), _p(dV), m, n)
    U, V = from_dev(dU, (m, k)), from_dev(dV, (n, k))
    assert np.all(np.diff(S) <= 0)
    assert np.abs(S - s_ref).max() <= 1e-12 * s_ref[0]
    big = s_ref > 1e-9 * s_ref[0]
    assert np.abs(S[big] / s_ref[big] - 1).max() < 1e-9
    assert np.abs((U * S) @ V.conj().T - X).max() < 1e-12 * s_ref[0]
    assert np.abs(U.conj().T @ U - np.eye(k)).max() < 1e-12
    assert np.abs(V.conj().T @ V - np.eye(k)).max() < 1e-12


def test_svd_rank_deficient(gpu_ctx):
    rng = np.random.default_rng(5)
    X = crand(rng, 40, 6) @ crand(rng, 6, 30)            # rank 6
    X[:, 3] = 0
    S = np.zeros(30)
    dX, dU, dV = to_dev(X), empty_dev((40, 30)), empty_dev((30, 30))
    _call(gpu_ctx, "mpsb_op_svd", _p(dX), _p(dU), S.ctypes.data_as(C.POINTER(C.c_double)), _p(dV), 40, 30)
    U, V = from_dev(dU, (40, 30)), from_dev(dV, (30, 30))
    s_ref = np.linalg.svd(X, compute_uv=False)
    assert np.abs(S - s_ref).max() < 1e-12 * s_ref[0]
    assert np.abs((U[:, :6] * S[:6]) @ V[:, :6].conj().T - X).max() < 1e-12 * s_ref[0]


SHAPES = [  # chiL, d, chiR, wL, wR, chi0
    (1, 2, 2, 1, 4, 2), (4, 2, 8, 4, 4, 8), (32, 2, 32, 4, 4, 32), (17, 3, 29, 5, 3, 23),
    (128, 4, 128, 8, 8, 128), (64, 4, 128, 6, 6, 100),
]


@pytest.mark.parametrize("shape", SHAPES)
def test_prod_AOR_and_update_re(gpu_ctx, shape):
    chiL, d, chiR, wL, wR, chiR0 = shape
    rng = np.random.default_rng(sum(shape))
    A, O, Rr = crand(rng, chiL, d, chiR), crand(rng, wL, d, wR, d), crand(rng, chiR, wR, chiR0)
    ref = R.prod_AOR(A, O, Rr)
    dA, dO, dR, dAOR = to_dev(A), to_dev(O), to_dev(Rr), empty_dev(ref.shape)
    _call(gpu_ctx, "mpsb_op_prod_AOR", _p(dA), _p(dO), _p(dR), _p(dAOR), chiL, d, chiR, wL, wR, chiR0)
    assert relerr(from_dev(dAOR, ref.shape), ref) < TOL
    # prod_LR!(A0, L, AOR) and update_re!(env, A0, AOR)
    chiL0 = max(1, chiL - 1)
    L = crand(rng, chiL, wL, chiL0)
    a0_ref = R.prod_LR(L, ref)
    dL, dA0 = to_dev(L), empty_dev(a0_ref.shape)
    _call(gpu_ctx, "mpsb_op_prod_LR_3_4", _p(dL), _p(dAOR), _p(dA0), chiL, wL, chiL0, d, chiR0)
    assert relerr(from_dev(dA0, a0_ref.shape), a0_ref) < TOL
    env_ref = R.update_re(a0_ref, ref)
    denv = empty_dev(env_ref.shape)
    _call(gpu_ctx, "mpsb_op_update_re", _p(dA0), _p(dAOR), _p(denv), chiL, wL, d, chiR0, chiL0)
    assert relerr(from_dev(denv, env_ref.shape), env_ref) < TOL


@pytest.mark.parametrize("shape", SHAPES)
def test_prod_AOL_and_update_le(gpu_ctx, shape):
    chiL, d, chiR, wL, wR, chiL0 = shape
    rng = np.random.default_rng(3 * sum(shape))
    A, O, L = crand(rng, chiL, d, chiR), crand(rng, wL, d, wR, d), crand(rng, chiL, wL, chiL0)
    ref = R.prod_AOL(A, O, L)
    dA, dO, dL, dAOL = to_dev(A), to_dev(O), to_dev(L), empty_dev(ref.shape)
    _call(gpu_ctx, "mpsb_op_prod_AOL", _p(dA), _p(dO), _p(dL), _p(dAOL), chiL, d, chiR, wL, wR, chiL0)
    assert relerr(from_dev(dAOL, ref.shape), ref) < TOL
    chiR0 = max(1, chiR - 2)
    Rr = crand(rng, chiR, wR, chiR0)
    a0_ref = R.prod_LR(ref, Rr)
    dR, dA0 = to_dev(Rr), empty_dev(a0_ref.shape)
    _call(gpu_ctx, "mpsb_op_prod_LR_4_3", _p(dAOL), _p(dR), _p(dA0), chiL0, d, chiR, wR, chiR0)
    assert relerr(from_dev(dA0, a0_ref.shape), a0_ref) < TOL
    env_ref = R.update_le(a0_ref, ref)
    denv = empty_dev(env_ref.shape)
    _call(gpu_ctx, "mpsb_op_update_le", _p(dA0), _p(dAOL), _p(denv), chiL0, d, chiR, wR, chiR0)
    assert relerr(from_dev(denv, env_ref.shape), env_ref) < TOL
