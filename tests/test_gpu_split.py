"""The int8-sliced tensor-core complex GEMM (tcgen05 kind::i8) and the split-precision sweeps.

* small-integer operands are represented exactly by the first slice, so the sliced GEMM must
  equal the exact product bit for bit (checks every index of the slicing, TMA, MMA and epilogue);
* random operands: the error against numpy's FP64 product stays inside the scheme's bound
  2^(-7 S) x 2K x max|A| max|B| (S slices), over shapes off the tile grid, conjugates, strides,
  alpha / beta and zero rows;
* the RK4 density-matrix step with split contractions stays within 1e-8 of the FP64 step on
  every observable (Tr rho, <sigma_ee_i>, <sigma+_i sigma-_j>).
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import crand, empty_dev, from_dev, to_dev

pytestmark = pytest.mark.gpu


def zgemm(ctx, A, B, C_init=None, conjA=False, conjB=False, transA=False, transB=False, alpha=1.0, beta=0.0,
          slices=6):
    """C = alpha op(A) op(B) + beta C through mpsb_op_zgemm; op folds transposes into strides."""
    from mpsb200 import _lib
    Ah, Bh = np.asarray(A), np.asarray(B)
    if transA:   # A is stored as A^T (K x M), column-major
        K, M = Ah.shape
        a_m, a_k = K, 1
    else:
        M, K = Ah.shape
        a_m, a_k = 1, M
    if transB:   # B stored as B^T (N x K)
        N = Bh.shape[0]
        b_k, b_n = N, 1
    else:
        N = Bh.shape[1]
        b_k, b_n = 1, K
    dA, dB = to_dev(Ah), to_dev(Bh)
    dC = to_dev(C_init) if C_init is not None else empty_dev((M, N))
    al = (C.c_double * 2)(np.real(alpha), np.imag(alpha))
    be = (C.c_double * 2)(np.real(beta), np.imag(beta))
    _lib.call("mpsb_op_zgemm", ctx.h, M, N, K, C.c_void_p(dA.data_ptr()), a_m, a_k, int(conjA),
              C.c_void_p(dB.data_ptr()), b_k, b_n, int(conjB), C.c_void_p(dC.data_ptr()), 1, M, al, be, slices)
    ctx.sync()
    return from_dev(dC, (M, N))


def op(X, conj, trans):
    Y = X.T if trans else X
    return Y.conj() if conj else Y


@pytest.mark.parametrize("slices", [3, 6, 7])
@pytest.mark.parametrize("shape", [(128, 32, 64), (200, 77, 333), (37, 300, 16)])
def test_small_integers_exact(gpu_ctx, slices, shape):
    M, N, K = shape
    rng = np.random.default_rng(M + N + K + slices)
    A = (rng.integers(-60, 61, (M, K)) + 1j * rng.integers(-60, 61, (M, K))).astype(np.complex128)
    B = (rng.integers(-60, 61, (K, N)) + 1j * rng.integers(-60, 61, (K, N))).astype(np.complex128)
    got = zgemm(gpu_ctx, A, B, slices=slices)
    assert np.array_equal(got, A @ B)


@pytest.mark.parametrize("slices", [4, 5, 6, 7])
@pytest.mark.parametrize("conjA,conjB,transA,transB", [(False, False, False, False), (True, False, True, False),
                                                       (False, True, False, True), (True, True, False, False)])
def test_random_within_bound(gpu_ctx, slices, conjA, conjB, transA, transB):
    rng = np.random.default_rng(slices * 7 + conjA + 2 * conjB)
    M, N, K = 300, 190, 520
    A = crand(rng, K, M) if transA else crand(rng, M, K)
    B = crand(rng, N, K) if transB else crand(rng, K, N)
    A[3] = 0.0   # a zero row / column of the stored operand
    Cin = crand(rng, M, N)
    alpha, beta = 0.7 - 0.2j, 0.3 + 0.5j
    got = zgemm(gpu_ctx, A, B, Cin, conjA, conjB, transA, transB, alpha, beta, slices)
    want = alpha * (op(A, conjA, transA) @ op(B, conjB, transB)) + beta * Cin
    bound = 4.0 * 2.0 ** (-7 * slices) * 2 * K * np.abs(A).max() * np.abs(B).max() * abs(alpha)
    assert np.abs(got - want).max() <= bound + 1e-13 * np.abs(want).max()


def test_wide_dynamic_range_rows(gpu_ctx):
    """Rows and columns scaled over 1e-200..1e200: the per-row / per-column exponents carry it."""
    rng = np.random.default_rng(3)
    M, N, K = 256, 96, 128
    ra = 10.0 ** rng.uniform(-200, 200, M)
    cb = 10.0 ** rng.uniform(-100, 100, N)
    A = crand(rng, M, K) * ra[:, None]
    B = crand(rng, K, N) * cb[None, :]
    got = zgemm(gpu_ctx, A, B, slices=6)
    want = A @ B
    scale = np.outer(ra, cb) * np.sqrt(K) * 4
    assert np.all(np.abs(got - want) <= 2.0 ** -38 * scale * 8)


def test_fp64_path_of_the_op(gpu_ctx):
    rng = np.random.default_rng(9)
    A, B = crand(rng, 70, 90), crand(rng, 90, 50)
    got = zgemm(gpu_ctx, A, B, slices=0)
    assert np.abs(got - A @ B).max() <= 1e-12 * np.abs(A @ B).max()


def _density_run(ctx, slices, na, chi, steps, rho_sites=None, dt=0.005):
    import mpsb200 as K
    from mpsb200 import drivers as GDR
    from mpsb200 import models as GM
    ctx.set_precision(slices, 1)   # every sweep GEMM on the chosen path
    p = GM.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    rho = K.MPS.from_sites(rho_sites, ctx) if rho_sites is not None else None
    b = GDR.DensityBuffers(p, chi, dt, 8, ctx, rho)
    obs = []
    for _ in range(steps):
        b.step()
        obs.append(b.observables(pairs=((0, 1), (na // 2 - 1, na // 2))))
    ctx.sync()
    return obs, b.rho.sites()


def _obs_err(a, b):
    return max(max(abs(x[0] - y[0]), np.abs(x[1] - y[1]).max(), np.abs(x[2] - y[2]).max()) for x, y in zip(a, b))


def test_split_rk4_density_matches_fp64():
    """Physical start (all-down rho, N=10, chi=32, truncated): the split step stays within 1e-8
    of the FP64 step on every observable over 8 steps, and differs from it (the path is taken)."""
    import mpsb200 as K
    c64, c6 = K.Context(0), K.Context(0)
    try:
        o64, s64 = _density_run(c64, 0, 10, 32, 8)
        o6, s6 = _density_run(c6, 6, 10, 32, 8)
    finally:
        c64.close()
        c6.close()
    err = _obs_err(o6, o64)
    assert err <= 1e-8, err
    assert any(np.abs(a - b).max() > 0 for a, b in zip(s6, s64))


def test_split_rk4_random_start_fidelity():
    """Random chi=16 MPS expanded to chi=64 (the precision configuration's start, scaled down):
    fidelity with the FP64 state and observables relative to their scale after 4 steps."""
    import mpsb200 as K
    from oracle import mps_ref as R

    from gpu_util import fidelity
    rng = np.random.default_rng(60)
    rho, _ = R.mpsrandom(10, 16, 4, rng)
    R.normalize_lo_(rho)
    start = R.expandmps(rho, 64)[0]
    c64, c6 = K.Context(0), K.Context(0)
    try:
        o64, s64 = _density_run(c64, 0, 10, 64, 4, start)
        o6, s6 = _density_run(c6, 6, 10, 64, 4, start)
    finally:
        c64.close()
        c6.close()
    scale = max(max(abs(x[0]), np.abs(x[1]).max(), np.abs(x[2]).max()) for x in o64)
    assert _obs_err(o6, o64) <= 1e-8 * scale
    assert 1 - fidelity(s6, s64) <= 1e-10


def test_bounded_wait_runs_out_and_the_context_recovers(gpu_ctx):
    """Failure detection without a fault: a device wait on a barrier nothing arrives on gives up
    after 50 ms, the call reports the timeout through the error word, and the same context then
    computes a sliced GEMM correctly."""
    import time

    from mpsb200 import _lib
    t0 = time.perf_counter()
    with pytest.raises(_lib.MpsbError) as e:
        _lib.call("mpsb_wait_selftest", gpu_ctx.h, 0.05)
    assert e.value.status == -3 and "timed out" in str(e.value) and "wait self-test" in str(e.value)
    assert time.perf_counter() - t0 < 5.0
    rng = np.random.default_rng(12)
    A, B = crand(rng, 96, 64), crand(rng, 64, 40)
    got = zgemm(gpu_ctx, A, B, slices=6)
    assert np.abs(got - A @ B).max() <= 4 * 2.0 ** -42 * 128 * np.abs(A).max() * np.abs(B).max()
