"""Full-sweep sum compressions and the Arnoldi step (the §f1 row) on the GPU against the oracle."""
import numpy as np
import pytest

from gpu_util import fidelity, relerr
from oracle import dense as D
from oracle import models as OM
from oracle import mps_ref as R

pytestmark = pytest.mark.gpu


def _sites_close(gpu_mps, ref_sites, tol):
    for k, (a, b) in enumerate(zip(gpu_mps.sites(), ref_sites)):
        assert relerr(a, b) < tol, "site %d: %.3e" % (k, relerr(a, b))


def _randoms(na, chi, d, n, seed):
    rng = np.random.default_rng(seed)
    out = [R.mpsrandom(na, chi, d, rng) for _ in range(n)]
    return [m for m, _ in out], out[0][1]


@pytest.mark.parametrize("sweeps", [1, 2])
def test_compress_sum_var_apply_H_full_sweeps(gpu_ctx, sweeps):
    """compress_sum_var_apply_H! (src/compression.jl:805-887): two plain terms + H term."""
    import mpsb200 as K
    na, chi = 8, 8
    terms, dims = _randoms(na, chi, 2, 4, 31)
    p = OM.SpinChain(na, omega=0.5)
    H = OM.sm_hamiltonian(p, 0.5, 0.05, 0.0)
    wl = [1] + [4] * (na - 1) + [1]
    coef = [0.4 - 0.1j, -0.3j, 1.0]
    A0 = R.copy_mps(terms[3])
    eop = R.build_env(dims, dims, wl)
    R.compress_sum_var_apply_H_(A0, eop, coef, terms[:3], H, sweeps)
    g = [K.MPS.from_sites(t, gpu_ctx) for t in terms]
    gA0 = g[3].clone()
    geop = K.build_env(dims, dims, wl, gpu_ctx)
    K.compress_sum_var_apply_H_(gA0, geop, coef, g[:3], K.MPO.from_sites(H, gpu_ctx), sweeps)
    _sites_close(gA0, A0, 1e-10)


def test_compress_sum_var(gpu_ctx):
    """compress_sum_var (src/compression.jl:496-565): three plain terms, guess = first term."""
    import mpsb200 as K
    na, chi = 9, 8
    terms, dims = _randoms(na, chi, 2, 3, 32)
    coef = [0.3 - 0.2j, 1.1, -0.7j]
    ref = R.compress_sum_var(R.copy_mps(terms[0]), coef, terms, 1)
    g = [K.MPS.from_sites(t, gpu_ctx) for t in terms]
    out = K.compress_sum_var(g[0], coef, g, 1)
    _sites_close(out, ref, 1e-10)
    with pytest.raises(K.MpsbError):   # the output must not be one of the terms
        from mpsb200 import _lib
        import ctypes as C
        cb = np.asarray(coef, dtype=np.complex128).view(np.float64)
        arr = (C.c_void_p * 3)(*[m.h.value for m in g])
        _lib.call("mpsb_compress_sum_var", gpu_ctx.h, g[0].h, g[0].h,
                  cb.ctypes.data_as(C.POINTER(C.c_double)), 3, arr, 1)


@pytest.mark.parametrize("na,chi,numv", [(8, 16, 4), (10, 8, 3)])
def test_arnoldi_expm_matches_oracle(gpu_ctx, na, chi, numv):
    """Arnoldi_expm! (src/timeevolution.jl:88-119): Krylov coefficients and the new state."""
    import mpsb200 as K
    dt = 0.02
    p = OM.SpinChain(na, omega=0.5)
    A = OM.sm_hamiltonian(p, 0, dt, 0.0)
    rng = np.random.default_rng(33)
    psi, dims = R.mpsrandom(na, chi, 2, rng)
    R.normalize_lo_(psi)
    wl = [1] + [4] * (na - 1) + [1]
    rhov = [R.copy_mps(psi) for _ in range(numv)]
    coef = R.Arnoldi_expm_(A, rhov, numv, None, R.build_env(dims, dims, wl))
    gpsi = K.MPS.from_sites(psi, gpu_ctx)
    grhov = [gpsi.clone() for _ in range(numv)]
    gcoef = K.Arnoldi_expm_(K.MPO.from_sites(A, gpu_ctx), grhov, numv, None,
                            K.build_env(dims, dims, wl, gpu_ctx))
    assert np.abs(np.asarray(gcoef) - coef).max() < 1e-10
    got, want = grhov[0].sites(), rhov[0]
    if chi >= 2 ** (na // 2):   # full bond dimension: the states themselves
        assert np.abs(D.mps_to_dense(got) - D.mps_to_dense(want)).max() < 1e-10
    else:
        _sites_close(grhov[0], want, 1e-9)
    assert 1 - fidelity(got, want) < 1e-12


def _tfi_mpo(na, J=1.0, h=0.7):
    I, Z, X = np.eye(2), np.diag([1.0, -1.0]), np.array([[0.0, 1.0], [1.0, 0.0]])
    W = np.zeros((3, 2, 3, 2), dtype=np.complex128)
    W[0, :, 0, :] = I
    W[1, :, 0, :] = Z
    W[2, :, 0, :] = -h * X
    W[2, :, 1, :] = -J * Z
    W[2, :, 2, :] = I
    return [W[2:3].copy()] + [W.copy() for _ in range(na - 2)] + [W[:, :, 0:1].copy()]


def _real_lo_guess(na, chi, seed):
    rng = np.random.default_rng(seed)
    A, dims = R.mpsrandom(na, chi, 2, rng)
    A = [a.real.astype(np.complex128) for a in A]
    R.leftorthonormalizationQR_(A)
    return A, dims


@pytest.mark.parametrize("na,chi,sweeps", [(8, 16, 3), (12, 8, 2)])
def test_ground_state_search_matches_oracle(gpu_ctx, na, chi, sweeps):
    """ground_state_search! (src/groundstate.jl:67-147): eigenvalue and state (full and truncated
    bond dimension); at full bond dimension also the exact ground energy."""
    import mpsb200 as K
    from oracle import groundstate as G
    H = _tfi_mpo(na)
    A, _ = _real_lo_guess(na, chi, 2)
    gA = K.MPS.from_sites(A, gpu_ctx)
    ae_ref = G.ground_state_search_(A, H, sweeps, 10.0, 1e-12)
    ae = K.ground_state_search_(gA, K.MPO.from_sites(H, gpu_ctx), sweeps, 10.0, 1e-12)
    assert abs(ae - ae_ref) < 1e-10 * abs(ae_ref)
    assert 1 - fidelity(gA.sites(), A) < 1e-10
    if chi >= 2 ** (na // 2):
        assert abs(ae - np.linalg.eigvalsh(D.mpo_to_dense(H))[0]) < 1e-10 * abs(ae)


def test_steady_state_search_matches_oracle(gpu_ctx):
    """steady_state_search! (src/steadystate.jl:6-86) for a real non-Hermitian L: the lowest
    eigenvalue of L^dagger L (zero at a steady state) and its state."""
    import mpsb200 as K
    from oracle import groundstate as G
    na = 6
    L = _tfi_mpo(na, J=1.0, h=0.4)
    for o in L:                              # a longitudinal field: non-degenerate lowest level
        o[o.shape[0] - 1, :, 0, :] += -0.3 * np.diag([1.0, -1.0])
    for o in L[1:-1]:                        # non-Hermitian: an asymmetric hopping term
        o[1, :, 0, :] = np.array([[0.0, 1.3], [0.2, 0.0]])
    Lconj = [np.conj(o.transpose(0, 3, 2, 1)) for o in L]
    A, _ = _real_lo_guess(na, 8, 3)
    gA = K.MPS.from_sites(A, gpu_ctx)
    ae_ref = G.steady_state_search_(A, L, Lconj, 3, 10.0, 1e-12)
    ae = K.steady_state_search_(gA, K.MPO.from_sites(L, gpu_ctx), K.MPO.from_sites(Lconj, gpu_ctx), 3, 10.0, 1e-12)
    Ld = D.mpo_to_dense(L)
    assert abs(ae - ae_ref) < 1e-10 * max(1.0, abs(ae_ref))
    assert abs(ae - np.linalg.eigvalsh(Ld.conj().T @ Ld)[0]) < 1e-9 * max(1.0, abs(ae))
    assert 1 - fidelity(gA.sites(), A) < 1e-10


@pytest.mark.parametrize("dmax,tol", [(16, 1e-15), (6, 1e-4), (9, 1e-12)])
def test_compression_svd_matches_oracle(gpu_ctx, dmax, tol):
    """compressionSVD! (src/compression.jl:1280-1312): new bond dims, the errors and entropies,
    and the truncated state (singular vectors are unique only up to phases)."""
    import mpsb200 as K
    rng = np.random.default_rng(40)
    A, dims = R.mpsrandom(9, 16, 2, rng)
    A[-1] = A[-1] * 0.9
    B = R.copy_mps(A)
    eg, et, ee = R.compressionSVD_(B, dmax, tol)
    gnew, geg, get, gee = K.compressionSVD_(K.MPS.from_sites(A, gpu_ctx), dmax, tol)
    assert gnew.dims == [1] + [b.shape[2] for b in B]
    assert abs(geg - eg) < 1e-12
    assert np.abs(get - et).max() < 1e-12
    assert np.abs(gee - ee).max() < 1e-10
    assert 1 - fidelity(gnew.sites(), B) < 1e-12


@pytest.mark.parametrize("dlim,tol,sweeps", [(16, 1e-14, 2), (6, 1e-10, 2), (12, 1e-3, 1)])
def test_two_site_compression_matches_oracle(gpu_ctx, dlim, tol, sweeps):
    """compress_var_apply_H_two_site / compress_var_two_site (the two-site SVD sweeps): adapted
    bond dims and the compressed state (singular vectors are unique only up to phases)."""
    import mpsb200 as K
    na = 9
    rng = np.random.default_rng(50)
    A, dims = R.mpsrandom(na, 8, 2, rng)
    H = OM.sm_hamiltonian(OM.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    dd = list(dims)
    ref = R.compress_var_apply_H_two_site(R.copy_mps(A), A, H, sweeps, tol, dd, dlim)
    gA = K.MPS.from_sites(A, gpu_ctx)
    gd = list(dims)
    got = K.compress_var_apply_H_two_site(gA, gA, K.MPO.from_sites(H, gpu_ctx), sweeps, tol, gd, dlim)
    assert gd == dd and got.dims == dd
    assert 1 - fidelity(got.sites(), ref) < 1e-10
    assert abs(R.scal_prod(got.sites(), got.sites()) / R.scal_prod(ref, ref) - 1) < 1e-10
    # the plain (operator-free) form
    ident = [np.eye(2, dtype=np.complex128).reshape(1, 2, 1, 2)] * na
    dd2 = list(dims)
    ref2 = R.compress_var_apply_H_two_site(R.copy_mps(A), A, ident, 1, 1e-14, dd2, dlim)
    gd2 = list(dims)
    got2 = K.compress_var_two_site(gA, gA, 1, 1e-14, gd2, dlim)
    assert gd2 == dd2 and 1 - fidelity(got2.sites(), ref2) < 1e-10


def test_two_site_guess_with_bonds_above_the_dims_rule(gpu_ctx):
    """A guess whose bonds exceed the dims rule ([1,2,8,8,8,8,8,2,1] at d=2): the pairs next to
    such a bond may need more than the rule allows, which the sweep scratch provides (nothing is
    cut below the truncation rule); bonds and state equal the oracle's."""
    import mpsb200 as K
    na = 8
    rng = np.random.default_rng(77)
    A, dims = R.mpsrandom(na, 16, 2, rng)          # the full-rank target [1,2,4,8,16,8,4,2,1]
    gdims = [1, 2, 8, 8, 8, 8, 8, 2, 1]
    guess = [0.3 * R.crandn(rng, gdims[k], 2, gdims[k + 1]) for k in range(na)]
    ident = [np.eye(2, dtype=np.complex128).reshape(1, 2, 1, 2)] * na
    dd = list(gdims)
    ref = R.compress_var_apply_H_two_site(R.copy_mps(guess), A, ident, 2, 1e-14, dd, 64)
    gd = list(gdims)
    got = K.compress_var_two_site(K.MPS.from_sites(guess, gpu_ctx), K.MPS.from_sites(A, gpu_ctx), 2, 1e-14, gd, 64)
    assert gd == dd and got.dims == dd
    assert all(x <= y for x, y in zip(gd, dims))
    assert 1 - fidelity(got.sites(), A) < 1e-12 and 1 - fidelity(got.sites(), ref) < 1e-12


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("with_h", [True, False])
@pytest.mark.parametrize("dlim,tol", [(16, 1e-14), (5, 1e-6)])
def test_two_site_sum_compression_matches_oracle(gpu_ctx, mode, with_h, dlim, tol):
    """compress_sum_var_apply_H_two_site with its _left / _right half sweeps, and
    compress_sum_var_two_site: three complex-weighted terms (the last through H when given),
    at full bond dimension and truncated; bond dims, norm and fidelity against the oracle."""
    import mpsb200 as K
    na = 7
    rng = np.random.default_rng(60 + mode)
    terms = [R.mpsrandom(na, 4, 2, rng)[0] for _ in range(3)]
    coef = [0.7 - 0.2j, -0.4 + 0.9j, 1.3 + 0.1j]
    H = OM.sm_hamiltonian(OM.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    guess, dims = R.mpsrandom(na, 8, 2, rng)
    if mode == 2:
        R.rightorthogonalizeQR_(guess)
    dd = list(dims)
    ref = R.compress_sum_var_apply_H_two_site(R.copy_mps(guess), coef, terms, H if with_h else None, 2, tol, dd,
                                              dlim, mode)
    gterms = [K.MPS.from_sites(t, gpu_ctx) for t in terms]
    gguess = K.MPS.from_sites(guess, gpu_ctx)
    gd = list(dims)
    if mode == 0 and not with_h:
        got = K.compress_sum_var_two_site(gguess, coef, gterms, 2, tol, gd, dlim)
    else:
        fn = {0: K.compress_sum_var_apply_H_two_site, 1: K.compress_sum_var_apply_H_two_site_left,
              2: K.compress_sum_var_apply_H_two_site_right}[mode]
        gH = K.MPO.from_sites(H, gpu_ctx) if with_h else None   # None: every term plain
        got = fn(gguess, coef, gterms, gH, 2, tol, gd, dlim)
    assert gd == dd and got.dims == dd
    assert 1 - fidelity(got.sites(), ref) < 1e-10
    assert abs(R.scal_prod(got.sites(), got.sites()) / R.scal_prod(ref, ref) - 1) < 1e-10


def test_two_site_sum_terms_of_different_bond_dims(gpu_ctx):
    """The stages of a two-site RK4 step sum MPSs whose bonds differ: each plain term keeps
    its own environments."""
    import mpsb200 as K
    na = 7
    rng = np.random.default_rng(71)
    terms = [R.mpsrandom(na, dm, 2, rng)[0] for dm in (2, 8, 4)]
    coef = [0.3 + 0.4j, -1.1, 0.5j]
    H = OM.sm_hamiltonian(OM.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    guess, dims = R.mpsrandom(na, 4, 2, rng)
    for mode in (0, 1):
        dd = list(dims)
        ref = R.compress_sum_var_apply_H_two_site(R.copy_mps(guess), coef, terms, H, 1, 1e-10, dd, 12, mode)
        gd = list(dims)
        fn = K.compress_sum_var_apply_H_two_site if mode == 0 else K.compress_sum_var_apply_H_two_site_left
        got = fn(K.MPS.from_sites(guess, gpu_ctx), coef, [K.MPS.from_sites(t, gpu_ctx) for t in terms],
                 K.MPO.from_sites(H, gpu_ctx), 1, 1e-10, gd, 12)
        assert gd == dd
        assert 1 - fidelity(got.sites(), ref) < 1e-10


@pytest.mark.parametrize("dlim,tol", [(16, 1e-14), (6, 1e-10)])
def test_two_site_rk4_step_matches_oracle(gpu_ctx, dlim, tol):
    """RK4stp_apply_H_half_full_two_site: three steps with adapting bonds (and at the full bond
    dimension, where the oracle equals the dense RK4 map)."""
    import mpsb200 as K
    na, dt = 8, 0.01
    rng = np.random.default_rng(81)
    psi, dims = R.mpsrandom(na, 4, 2, rng)
    p = OM.SpinChain(na, omega=0.5)
    H = [OM.sm_hamiltonian(p, 1, dt / 2, 0), OM.sm_hamiltonian(p, 0, 1, dt / 2), OM.sm_hamiltonian(p, 1, dt / 2, dt)]
    gH = [K.MPO.from_sites(h, gpu_ctx) for h in H]
    g = K.MPS.from_sites(psi, gpu_ctx)
    dd, gd = list(dims), list(dims)
    for _ in range(3):
        psi = R.RK4stp_apply_H_half_full_two_site(dt, H, psi, tol, dd, dlim)
        g = K.RK4stp_apply_H_half_full_two_site(dt, gH, g, tol, gd, dlim)
        assert gd == dd and g.dims == dd
        assert 1 - fidelity(g.sites(), psi) < 1e-10
        assert abs(R.scal_prod(g.sites(), g.sites()) / R.scal_prod(psi, psi) - 1) < 1e-10


def test_allocating_forms_match_oracle(gpu_ctx):
    """The reference's allocating compressions (compress_var, compress_var_apply_H and its
    _left / _right, compress_sum_var_apply_H and its _left / _right) return a new MPS equal to
    the in-place forms run on fresh buffers."""
    import mpsb200 as K
    na = 6
    rng = np.random.default_rng(91)
    Ain, dims = R.mpsrandom(na, 4, 2, rng)
    terms = [R.mpsrandom(na, 4, 2, rng)[0] for _ in range(3)]
    coef = [0.8, -0.3 + 0.2j, 0.6 - 0.1j]
    H = OM.sm_hamiltonian(OM.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    w = [h.shape[0] for h in H] + [1]
    g = lambda x: K.MPS.from_sites(x, gpu_ctx)     # noqa: E731
    gAin, gterms, gH = g(Ain), [g(t) for t in terms], K.MPO.from_sites(H, gpu_ctx)

    def oracle(fn, *args, plain=0):
        A0 = R.copy_mps(Ain)
        envop = R.build_env(dims, dims, w)
        env = [R.build_env(dims, dims) for _ in range(plain)]
        fn(A0, *([env] if plain or fn in (R.compress_sum_var_apply_H_right_, R.compress_sum_var_apply_H_left_) else []),
           envop, *args)
        return A0

    cases = [
        (K.compress_var(gAin, gterms[0], 2), R.compress_sum_var(R.copy_mps(Ain), [1.0], [terms[0]], 2)),
        (K.compress_var_apply_H(gAin, gterms[0], gH, 2), oracle(R.compress_var_apply_H_, Ain, terms[0], H, 2)),
        (K.compress_var_apply_H_left(gAin, gterms[0], gH), oracle(R.compress_var_apply_H_left_, Ain, terms[0], H)),
        (K.compress_var_apply_H_right(gAin, gterms[0], gH),   # the oracle's form wants a plain term: weight 0
         oracle(R.compress_sum_var_apply_H_right_, Ain, [0.0, 1.0], [terms[0], terms[0]], H, plain=1)),
        (K.compress_sum_var_apply_H(gAin, coef, gterms, gH, 2),
         oracle(R.compress_sum_var_apply_H_, coef, terms, H, 2)),
        (K.compress_sum_var_apply_H_left(gAin, coef, gterms, gH),
         oracle(R.compress_sum_var_apply_H_left_, Ain, coef, terms, H, plain=2)),
        (K.compress_sum_var_apply_H_right(gAin, coef, gterms, gH),
         oracle(R.compress_sum_var_apply_H_right_, Ain, coef, terms, H, plain=2)),
    ]
    for got, ref in cases:
        assert got.dims == dims
        assert 1 - fidelity(got.sites(), ref) < 1e-10
        assert abs(R.scal_prod(got.sites(), got.sites()) / R.scal_prod(ref, ref) - 1) < 1e-10
