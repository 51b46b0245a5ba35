"""Pins of the CPU oracle (no GPU): exact dense evolution, independent generators, op algebra."""
import numpy as np
import pytest

from oracle import dense as D
from oracle import drivers as DR
from oracle import models as M
from oracle import mps_ref as R

RNG = np.random.default_rng(1234)


def crand(*shape):
    return RNG.standard_normal(shape) + 1j * RNG.standard_normal(shape)


# ---------------------------------------------------------------- op algebra

def test_prod_AOR_matches_einsum():
    A, O, Rr = crand(3, 2, 5), crand(4, 2, 6, 2), crand(5, 6, 7)
    ref = np.einsum("asb,wtvs,bvc->awtc", A, O, Rr)
    assert np.allclose(R.prod_AOR(A, O, Rr), ref, rtol=0, atol=1e-12)


def test_prod_AOL_matches_einsum():
    A, O, L = crand(3, 2, 5), crand(4, 2, 6, 2), crand(3, 4, 7)
    ref = np.einsum("awx,asb,wtvs->xtbv", L.conj(), A, O)
    assert np.allclose(R.prod_AOL(A, O, L), ref, rtol=0, atol=1e-12)


def test_env_updates_match_einsum():
    AOR, A0 = crand(3, 4, 2, 5), crand(6, 2, 5)
    assert np.allclose(R.update_re(A0, AOR), np.einsum("awtc,xtc->awx", AOR, A0.conj()), atol=1e-12)
    AOL, B0 = crand(6, 2, 5, 4), crand(6, 2, 3)
    assert np.allclose(R.update_le(B0, AOL), np.einsum("xtbv,xty->bvy", AOL.conj(), B0), atol=1e-12)
    A, FL, FR = crand(3, 2, 5), crand(4, 3), crand(5, 4)
    AL = R.prod_LR(FL, A)
    assert np.allclose(AL, np.einsum("xa,asb->xsb", FL, A), atol=1e-12)
    C0 = crand(4, 2, 6)
    assert np.allclose(R.update_lenv(C0, AL), np.einsum("xsy,xsb->yb", C0.conj(), AL), atol=1e-12)
    assert np.allclose(R.update_lenv_nc(C0, AL), np.einsum("xsy,xsb->yb", C0, AL), atol=1e-12)
    AR = R.prod_LR(A, FR)
    D0 = crand(7, 2, 4)
    assert np.allclose(R.update_renv(D0, AR), np.einsum("asb,xsb->ax", AR, D0.conj()), atol=1e-12)


def test_qr_is_lapack_householder_convention():
    X = crand(12, 5)
    q, r = R.julia_qr(X)
    assert np.allclose(q.conj().T @ q, np.eye(5), atol=1e-13)
    assert np.allclose(q @ r, X, atol=1e-12)
    # zlarfg makes the diagonal of R real with sign -sign(Re alpha) on the first column
    assert np.allclose(np.imag(np.diag(r)), 0, atol=1e-14)
    assert np.sign(r[0, 0].real) == -np.sign(X[0, 0].real)


def test_rightorth_gives_right_orthonormal_site():
    A = crand(4, 2, 3)
    Q = R.rightorth_(A)
    m = R.jr(Q, 4, 6)
    assert np.allclose(m @ m.conj().T, np.eye(4), atol=1e-13)


def test_dims_rule_and_product_state():
    mps, dims = R.mpsgroundstate(10, 8, 2)
    assert dims == R.dims_rule(10, 8, 2) == [1, 2, 4, 8, 8, 8, 8, 8, 4, 2, 1]
    v = D.mps_to_dense(mps)
    e = np.zeros(2 ** 10)
    e[0] = 1
    assert np.allclose(v, e, atol=1e-14)


def test_mpo_algebra():
    p = M.SpinChain(5, omega=0.3)
    jr_, _ = M.jump_mpos(p)
    c = R.conj_mpo(jr_)
    prod = R.applyMPOtoMPO(jr_, c)
    Jd, Cd, Pd = (D.mpo_to_dense(x) for x in (jr_, c, prod))
    assert np.allclose(Cd, Jd.conj().T, atol=1e-13)
    assert np.allclose(Pd, Cd @ Jd, atol=1e-13)
    A, _ = R.mpsrandom(5, 4, 2, np.random.default_rng(3))
    out = R.applyMPOtoMPS(A, jr_)
    assert np.allclose(D.mps_to_dense(out), Jd @ D.mps_to_dense(A), atol=1e-12)


# ---------------------------------------------------------------- generators

def _op_at(o, i, n, d=2):
    m = np.eye(1)
    for j in range(n):
        m = np.kron(m, o if j == i else np.eye(d))
    return m


def test_trajectory_generator_is_waveguide_heff():
    n, phi, om = 6, 0.5 * np.pi, 0.5
    p = M.SpinChain(n, k_wg=phi, omega=om)
    G = D.mpo_to_dense(M.sm_hamiltonian(p, 0, 1, 0.0))
    Heff = np.zeros((2 ** n, 2 ** n), complex)
    for i in range(n):
        Heff += -om * (_op_at(M.heg, i, n) + _op_at(M.hge, i, n))
        for j in range(n):
            Heff += -0.5j * np.exp(1j * phi * abs(i - j)) * _op_at(M.heg, i, n) @ _op_at(M.hge, j, n)
    assert np.abs(G - (-1j) * Heff).max() < 1e-13


def _dense_lindbladian(n, phi, om, gam, gam_eg, gam_phi):
    """Superoperator on the per-site-interleaved vec(rho) used by the MPS ([gg,ge,eg,ee] per site)."""
    D_ = 2 ** n
    sp = [_op_at(M.heg, i, n) for i in range(n)]
    sm = [_op_at(M.hge, i, n) for i in range(n)]
    see = [_op_at(M.hee, i, n) for i in range(n)]
    Heff = np.zeros((D_, D_), complex)
    for i in range(n):
        Heff += -om * (sp[i] + sm[i]) - 0.5j * (gam_eg + gam_phi) * see[i]
        for j in range(n):
            Heff += -0.5j * gam * np.exp(1j * phi * abs(i - j)) * sp[i] @ sm[j]
    I = np.eye(D_)
    Lsup = -1j * (np.kron(Heff, I) - np.kron(I, Heff.conj()))   # C-order vec: X rho Y -> X (x) Y^T
    for i in range(n):
        Lsup += gam_eg * np.kron(sm[i], sm[i].conj())
        Lsup += gam_phi * np.kron(see[i], see[i].conj())
        for j in range(n):
            Lsup += gam * np.cos(phi * abs(i - j)) * np.kron(sm[j], sm[i].conj())
    # reorder (a1..an, b1..bn) -> (a1 b1, ..., an bn)
    perm = [x for k in range(n) for x in (k, n + k)]
    T = Lsup.reshape([2] * (4 * n))
    T = T.transpose(perm + [2 * n + q for q in perm])
    return T.reshape(4 ** n, 4 ** n)


def test_density_generator_is_lindbladian():
    n, phi, om, gam_eg, gam_phi = 4, 0.5 * np.pi, 0.5, 0.1, 0.2
    p = M.SpinChain(n, k_wg=phi, omega=om, gam_eg=gam_eg, gam_phi=gam_phi)
    G = D.mpo_to_dense(M.construct_L_spin_model(p, 0, 1, 0.0))
    Lref = _dense_lindbladian(n, phi, om, 1.0, gam_eg, gam_phi)
    assert np.abs(G - Lref).max() < 1e-13
    G8 = D.mpo_to_dense(M.construct_L_spin_model(p, 0, 1, 0.0, w=8))
    assert np.abs(G8 - Lref).max() < 1e-13


# ---------------------------------------------------------------- dense pins

def test_rk4_trajectory_full_bond_matches_dense():
    n, dt = 6, 0.01
    p = M.SpinChain(n, omega=0.5)
    A, dims = R.mpsgroundstate(n, 8, 2)
    H = [M.sm_hamiltonian(p, 1, dt / 2, 0), M.sm_hamiltonian(p, 0, 1, dt / 2), M.sm_hamiltonian(p, 1, dt / 2, dt)]
    Hd = [D.mpo_to_dense(h) for h in H]
    psi = D.mps_to_dense(A)
    A1, A2, A3, A0 = (R.copy_mps(A) for _ in range(4))
    envop = R.build_env(dims, dims, [4] * (n + 1))
    e1, e2, e3 = (R.build_env(dims, dims) for _ in range(3))
    for _ in range(6):
        R.RK4stp_apply_H_half_(dt, H, A0, A, A1, A2, A3, e1, e2, e3, envop)
        psi = D.rk4_dense_step(*Hd, psi, dt)
        assert np.abs(D.mps_to_dense(A0) - psi).max() < 1e-13
        A = R.copy_mps(A0)
    # RK4 algebra: psi + dt/6 (k1 + 2k2 + 2k3 + k4) for the time-independent generator
    G = Hd[1]
    v = D.mps_to_dense(R.mpsgroundstate(n, 8, 2)[0])
    k1 = G @ v
    k2 = G @ (v + dt / 2 * k1)
    k3 = G @ (v + dt / 2 * k2)
    k4 = G @ (v + dt * k3)
    assert np.allclose(D.rk4_dense_step(*Hd, v, dt), v + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4), atol=1e-15)


def test_rk4_density_full_bond_matches_dense_and_keeps_trace():
    n, dt = 4, 0.005
    p = M.SpinChain(n, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    rho, obs = DR.run_density(p, 16, dt, 6, w=8, measure_int=1)
    L = [M.construct_L_spin_model(p, 1, dt / 2, 0, 8), M.construct_L_spin_model(p, 0, 1, dt / 2, 8),
         M.construct_L_spin_model(p, 1, dt / 2, dt, 8)]
    Ld = [D.mpo_to_dense(x) for x in L]
    v = D.mps_to_dense(R.mpsgroundstate(n, 16, 4)[0])
    for _ in range(6):
        v = D.rk4_dense_step(*Ld, v, dt)
    assert np.abs(D.mps_to_dense(rho) - v).max() < 1e-13
    for tr, _, _ in obs:
        assert abs(tr - 1) < 1e-13
    # hermiticity of rho: rho_ab = conj(rho_ba)
    Rm = v.reshape([2, 2] * n).transpose([2 * k for k in range(n)] + [2 * k + 1 for k in range(n)])
    Rm = Rm.reshape(2 ** n, 2 ** n)
    assert np.allclose(Rm, Rm.conj().T, atol=1e-14)


def test_trajectory_probability_identity():
    """p_coh + sum dt*p_jump = 1 + O(dt^2) (examples/spin_model_quantum_trajectory_rk4.jl:151)."""
    n, dt = 6, 0.01
    p = M.SpinChain(n, omega=0.5)
    r1 = np.concatenate([np.zeros(40), np.ones(10)])   # coherent, then the jump branch every step
    r2 = np.full(50, 0.3)
    rec = DR.run_trajectory(p, 8, dt, 50, r1, r2, measure_int=5)
    assert len(rec["jumps"]) == 10
    assert max(j[4] for j in rec["jumps"]) > 1e-3
    for (_, _, _, p_coh, p_sum) in rec["jumps"]:
        assert abs(p_coh + p_sum - 1) < 2e-4


@pytest.mark.parametrize("seed", [0])
def test_trajectory_runs_and_normalises(seed):
    p = M.SpinChain(8, omega=0.5)
    r1, r2 = DR.uniforms(seed, 30)
    rec = DR.run_trajectory(p, 8, 0.01, 30, r1, r2, measure_int=10)
    assert abs(R.norm_lo(rec["A"]) - 1) < 1e-12
    assert rec["e_pop"].shape == (4, 8)


def _arnoldi_dense(Ad, v0, numv):
    """Arnoldi_expm! (src/timeevolution.jl:88-119) restated on dense vectors, with the
    reference's own scalar conventions: scal_op_prod(m1, A, m2) = conj(<m1|A|m2>) (its left
    environments are stored conjugated, update_le = AOL' * A0, src/mps_base.jl:223-231) and
    scal_prod(m1, m2) = <m1|m2>."""
    import scipy.linalg
    sop = lambda a, b: np.conj(np.vdot(a, Ad @ b))
    v = [v0 / np.linalg.norm(v0)]
    Nm = np.eye(numv, dtype=complex)
    Hm = np.zeros((numv, numv), dtype=complex)
    Hm[0, 0] = sop(v[0], v[0])
    for jj in range(1, numv):
        w = Ad @ v[jj - 1] - sum(Hm[ll, jj - 1] * v[ll] for ll in range(jj))
        v.append(w / np.linalg.norm(w))
        Hm[jj, jj] = sop(v[jj], v[jj])
        for ll in range(jj):
            Hm[jj, ll] = sop(v[jj], v[ll])
            Hm[ll, jj] = sop(v[ll], v[jj])
            Nm[jj, ll] = np.vdot(v[jj], v[ll])
            Nm[ll, jj] = np.conj(Nm[jj, ll])
    coef = scipy.linalg.expm(np.linalg.solve(Nm, Hm))[:, 0]
    out = sum(c * x for c, x in zip(coef, v))
    return out / np.linalg.norm(out), coef


def test_arnoldi_expm_full_bond_matches_dense_restatement():
    """At full bond dimension every compression is exact, so the MPS Arnoldi step equals the
    same algorithm on dense vectors.  (Because scal_op_prod returns the conjugate matrix
    element, the reference's step is exp(A) psi only to first order in A for a general A.)"""
    import scipy.linalg
    na, dt = 5, 0.01
    p = M.SpinChain(na, omega=0.5)
    A = M.sm_hamiltonian(p, 0, dt, 0.0)
    Ad = D.mpo_to_dense(A)
    rng = np.random.default_rng(3)
    psi, dims = R.mpsrandom(na, 8, 2, rng)
    R.normalize_lo_(psi)
    for numv in (2, 4):
        rhov = [R.copy_mps(psi) for _ in range(numv)]
        envop = R.build_env(dims, dims, [1] + [4] * (na - 1) + [1])
        coef = R.Arnoldi_expm_(A, rhov, numv, None, envop)
        want, wcoef = _arnoldi_dense(Ad, D.mps_to_dense(psi), numv)
        got = D.mps_to_dense(rhov[0])
        assert np.abs(coef - wcoef).max() < 1e-10
        assert abs(np.linalg.norm(got) - 1) < 1e-12
        assert 1 - abs(np.vdot(want, got)) < 1e-12
        exact = scipy.linalg.expm(Ad) @ D.mps_to_dense(psi)
        assert 1 - abs(np.vdot(exact / np.linalg.norm(exact), got)) < 1e-2   # agrees to O(|A|) only


def test_compress_sum_var_full_bond_is_exact():
    """compress_sum_var (src/compression.jl:496-565) at full bond dimension reproduces the sum."""
    na = 5
    rng = np.random.default_rng(4)
    terms = [R.mpsrandom(na, 8, 2, rng)[0] for _ in range(3)]
    coef = [0.3 - 0.2j, 1.1, -0.7j]
    out = R.compress_sum_var(R.copy_mps(terms[0]), coef, terms, 1)
    want = sum(c * D.mps_to_dense(t) for c, t in zip(coef, terms))
    assert np.abs(D.mps_to_dense(out) - want).max() < 1e-12


def _tfi_mpo(na, J=1.0, h=0.7):
    """Transverse-field Ising chain -J sum Z Z - h sum X as a w=3 MPO O[wL, d_out, wR, d_in]."""
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


def test_lanczos_lowest_matches_eigh():
    from oracle import groundstate as G
    rng = np.random.default_rng(9)
    for n in (5, 60, 150):
        X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        Hm = X + X.conj().T
        th, x = G.lanczos_lowest(lambda v: Hm @ v, rng.standard_normal(n).astype(np.complex128), 1e-13)
        ev = np.linalg.eigvalsh(Hm)
        assert abs(th - ev[0]) < 1e-10 * max(1, abs(ev[0]))
        assert np.linalg.norm(Hm @ x - th * x) < 1e-8 * abs(th)


def test_effective_operators_are_product_mpo_contractions():
    """A_prod_LOR_eigs is prod_AOR then L (as stored, unconjugated) contracted; the two-operator
    A_prod_L_OO_R_eigs equals A_prod_LOR_eigs of the product MPO with fused bonds."""
    from oracle import groundstate as G
    rng = np.random.default_rng(10)
    c = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    Dl, d, Dr, w1, w1p, w2, w2p = 3, 2, 4, 2, 3, 3, 2
    L3, A, O, R3 = c(Dl, w1, Dl), c(Dl, d, Dr), c(w1, d, w1p, d), c(Dr, w1p, Dr)
    want = np.einsum("awx,awsy->xsy", L3, R.prod_AOR(A, O, R3)).ravel(order="F")
    assert np.abs(G.A_prod_LOR_eigs(L3, A.ravel(order="F"), O, R3) - want).max() < 1e-12
    O1, O2 = c(w1, d, w1p, d), c(w2, d, w2p, d)
    L4, R4 = c(Dl, w1, w2, Dl), c(Dr, w1p, w2p, Dr)
    P = G.product_mpo([O2], [O1])[0]
    got = G.A_prod_LOR_eigs(L4.reshape(Dl, w1 * w2, Dl, order="F"), A.ravel(order="F"), P,
                            R4.reshape(Dr, w1p * w2p, Dr, order="F"))
    assert np.abs(got - G.A_prod_L_OO_R_eigs(L4, A.ravel(order="F"), O1, O2, R4)).max() < 1e-12


def test_ground_state_search_tfi_matches_exact_diagonalisation():
    """ground_state_search! (src/groundstate.jl:67-147) on a real Hamiltonian from a real guess.
    (The reference contracts the conjugated-stored left environment without conjugation, so for
    complex states its local operator is not the true one; the port keeps that behaviour.)"""
    from oracle import groundstate as G
    na = 8
    H = _tfi_mpo(na)
    e0 = np.linalg.eigvalsh(D.mpo_to_dense(H))[0]
    A, _ = _real_lo_guess(na, 16, 1)
    ae = G.ground_state_search_(A, H, 3, 10.0, 1e-12)
    psi = D.mps_to_dense(A)
    assert abs(ae - e0) < 1e-10 * abs(e0)
    assert abs((psi.conj() @ D.mpo_to_dense(H) @ psi).real / np.vdot(psi, psi).real - e0) < 1e-10 * abs(e0)


def test_compression_svd_rule_and_exactness():
    """compressionSVD! (src/compression.jl:1280-1312): untruncated it reproduces the state (right
    canonical, err_glob = 1 - <psi|psi>); truncated, the dropped weights follow the rule."""
    rng = np.random.default_rng(12)
    A, dims = R.mpsrandom(8, 16, 2, rng)
    A[-1] = A[-1] * 0.8
    psi = D.mps_to_dense(A)
    B = R.copy_mps(A)
    eg, et, ee = R.compressionSVD_(B, 16, 1e-15)
    assert [b.shape[2] for b in B[:-1]] == dims[1:-1]
    assert abs(eg - (1 - 0.64)) < 1e-12 and np.abs(et).max() < 1e-14
    for b in B[1:]:   # right canonical
        m = b.reshape(b.shape[0], -1, order="F")
        assert np.abs(m @ m.conj().T - np.eye(b.shape[0])).max() < 1e-12
    got = D.mps_to_dense(B)
    assert abs(abs(np.vdot(got, psi)) / (np.linalg.norm(got) * np.linalg.norm(psi)) - 1) < 1e-12
    C = R.copy_mps(A)
    eg2, et2, ee2 = R.compressionSVD_(C, 5, 1e-3)
    assert max(c.shape[2] for c in C) <= 5
    assert np.all(et2 >= 0) and et2.max() > 0
    assert abs(ee2[-1] - ee[-1]) < 1e-12   # the first site processed sees the untruncated spectrum


def test_two_site_compression_exact_at_full_bond_dimension():
    """compress_var_apply_H_two_site (src/compression.jl:355-411, with a thin SVD for its
    undefined svdecon): with dlim at the full bond dimension it reproduces H*A, and the bonds
    grow from the guess's dims to what H*A needs."""
    na = 8
    rng = np.random.default_rng(3)
    A, dims = R.mpsrandom(na, 8, 2, rng)
    H = M.sm_hamiltonian(M.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    dd = list(dims)
    out = R.compress_var_apply_H_two_site(R.copy_mps(A), A, H, 2, 1e-14, dd, 16)
    want = D.mpo_to_dense(H) @ D.mps_to_dense(A)
    assert np.linalg.norm(D.mps_to_dense(out) - want) < 1e-12 * np.linalg.norm(want)
    assert dd == [1, 2, 4, 8, 16, 8, 4, 2, 1]


def _two_site_sum_case(na=6, seed=11):
    rng = np.random.default_rng(seed)
    terms = [R.mpsrandom(na, 4, 2, rng)[0] for _ in range(3)]
    coef = [0.7 - 0.2j, -0.4 + 0.9j, 1.3 + 0.1j]
    H = M.sm_hamiltonian(M.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    plain = sum(c * D.mps_to_dense(t) for c, t in zip(coef[:-1], terms[:-1]))
    with_h = plain + coef[-1] * (D.mpo_to_dense(H) @ D.mps_to_dense(terms[-1]))
    all_plain = plain + coef[-1] * D.mps_to_dense(terms[-1])
    return rng, terms, coef, H, with_h, all_plain


def test_two_site_sum_single_term_is_the_two_site_compression():
    na = 6
    rng = np.random.default_rng(4)
    A, dims = R.mpsrandom(na, 4, 2, rng)
    H = M.sm_hamiltonian(M.SpinChain(na, omega=0.5), 1.0, 0.05, 0.0)
    d1, d2 = list(dims), list(dims)
    a = R.compress_var_apply_H_two_site(R.copy_mps(A), A, H, 2, 1e-10, d1, 6)
    b = R.compress_sum_var_apply_H_two_site(R.copy_mps(A), [1.0], [A], H, 2, 1e-10, d2, 6)
    assert d1 == d2
    assert max(np.abs(x - y).max() for x, y in zip(a, b)) < 1e-14


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("with_h", [True, False])
def test_two_site_sum_exact_at_full_bond_dimension(mode, with_h):
    """compress_sum_var_apply_H_two_site (src/compression.jl:1072-1157), its _left / _right
    half sweeps (:1159-1276) and compress_sum_var_two_site (:574-648): from a guess at the
    full bond dimension (left canonical; right canonical for the L->R half sweep) and with no
    truncation, the result is the exact sum of the terms."""
    na = 6
    rng, terms, coef, H, want_h, want_p = _two_site_sum_case(na)
    guess, dims = R.mpsrandom(na, 8, 2, rng)
    if mode == 2:
        R.rightorthogonalizeQR_(guess)
    dd = list(dims)
    out = R.compress_sum_var_apply_H_two_site(guess, coef, terms, H if with_h else None, 1, 1e-14, dd, 16, mode)
    want = want_h if with_h else want_p
    assert np.linalg.norm(D.mps_to_dense(out) - want) < 1e-10 * np.linalg.norm(want)
    assert dd == [1, 2, 4, 8, 4, 2, 1]


def test_two_site_rk4_step_is_the_dense_rk4_map_at_full_bond_dimension():
    """RK4stp_apply_H_half_full_two_site (src/timeevolution.jl:208-215): from a left-canonical
    state at the full bond dimension and without truncation, three steps equal the dense RK4
    map, and the bonds stay at the full dims."""
    na, dt = 6, 0.01
    rng = np.random.default_rng(21)
    psi, dims = R.mpsrandom(na, 8, 2, rng)
    p = M.SpinChain(na, omega=0.5)
    H = [M.sm_hamiltonian(p, 1, dt / 2, 0), M.sm_hamiltonian(p, 0, 1, dt / 2), M.sm_hamiltonian(p, 1, dt / 2, dt)]
    Hd = [D.mpo_to_dense(h) for h in H]
    want = D.mps_to_dense(psi)
    dd = list(dims)
    for _ in range(3):
        psi = R.RK4stp_apply_H_half_full_two_site(dt, H, psi, 1e-14, dd, 16)
        want = D.rk4_dense_step(*Hd, want, dt)
        assert np.linalg.norm(D.mps_to_dense(psi) - want) < 1e-11 * np.linalg.norm(want)
    assert dd == [1, 2, 4, 8, 4, 2, 1]


def test_first_order_trajectory_step_agrees_with_rk4_to_second_order():
    """examples/spin_model_quantum_trajectory.jl (coherent step 1 - i dt H_eff through
    compress_var_apply_H!) against the RK4 example: the no-jump probabilities of the first
    steps agree to O(dt^2)."""
    from oracle import drivers as ODR
    p = M.SpinChain(8, omega=0.5)
    r1, r2 = np.zeros(3), np.zeros(3)            # no jumps
    a = ODR.run_trajectory(p, 16, 0.01, 3, r1, r2, measure_int=1, order=1)
    b = ODR.run_trajectory(p, 16, 0.01, 3, r1, r2, measure_int=1, order=4)
    assert np.all(np.abs(a["p_coh"] - b["p_coh"]) < 1e-3)
    assert np.abs(a["p_coh"] - b["p_coh"]).max() > 1e-6    # the first-order step is not unitary to O(dt^2)
