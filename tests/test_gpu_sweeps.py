"""Sweep / RK4 / observable / driver parity of the GPU engine with the oracle (via the C ABI)."""
import numpy as np
import pytest

from gpu_util import fidelity, perturbed_oracle_qr, relerr
from oracle import dense as D
from oracle import drivers as ODR
from oracle import models as OM
from oracle import mps_ref as R

pytestmark = pytest.mark.gpu


def _mps(K, sites, ctx):
    return K.MPS.from_sites(sites, ctx)


def _sites_close(gpu_mps, ref_sites, tol):
    for k, (a, b) in enumerate(zip(gpu_mps.sites(), ref_sites)):
        assert relerr(a, b) < tol, "site %d: %.3e" % (k, relerr(a, b))


def _random_lo(na, chi, d, seed):
    rng = np.random.default_rng(seed)
    A, dims = R.mpsrandom(na, chi, d, rng)
    return A, dims


def test_constructors_match(gpu_ctx):
    import mpsb200 as K
    for (na, dmax, d) in [(6, 8, 2), (10, 4, 2), (5, 16, 4)]:
        g, dims = K.mpsgroundstate(na, dmax, d, gpu_ctx)
        r, rdims = R.mpsgroundstate(na, dmax, d)
        assert dims == rdims
        _sites_close(g, r, 1e-14)
    rng1, rng2 = np.random.default_rng(11), np.random.default_rng(11)
    g, _ = K.mpsrandom(7, 8, 2, rng1, gpu_ctx)
    r, _ = R.mpsrandom(7, 8, 2, rng2)
    _sites_close(g, r, 1e-12)
    ge, _ = K.expandmps(g, 16)
    re_, _ = R.expandmps(r, 16)
    _sites_close(ge, re_, 1e-11)


@pytest.mark.parametrize("na,chi,d,w", [(8, 16, 2, 4), (10, 8, 2, 4), (6, 32, 4, 8)])
def test_compress_stages_match_oracle(gpu_ctx, na, chi, d, w):
    import mpsb200 as K
    A, dims = _random_lo(na, chi, d, 5)
    B, _ = _random_lo(na, chi, d, 6)
    rng = np.random.default_rng(9)
    H = [np.asarray(x) for x in (OM.sm_hamiltonian(OM.SpinChain(na, omega=0.4), 1, 0.05, 0.0) if d == 2 else
                                  OM.construct_L_spin_model(OM.SpinChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1), 1, 0.05, 0.0, w=w))]
    Hd = K.MPO.from_sites(H, gpu_ctx)
    wl = [1] + [h.shape[2] for h in H]
    gA, gB = _mps(K, A, gpu_ctx), _mps(K, B, gpu_ctx)
    # stage 1: compress_var_apply_H_left!
    out_ref = R.copy_mps(A)
    envop_ref = R.build_env(dims, dims, wl)
    R.compress_var_apply_H_left_(out_ref, envop_ref, A, A, H)
    gout = gA.clone()
    genvop = K.build_env(dims, dims, wl, gpu_ctx)
    K.compress_var_apply_H_left_(gout, genvop, gA, gA, Hd)
    _sites_close(gout, out_ref, 1e-10)
    # right / left sum stages with 1 and 3 plain terms, complex coefficients
    for right in (True, False):
        for coef in ([1.0, 0.025], [-1 / 3, 1 / 3 + 0.1j, 2 / 3, 0.2 - 0.3j]):
            numv = len(coef)
            terms_ref = [A, B, out_ref, A][:numv - 1] + [B]
            gterms = [gA, gB, gout, gA][:numv - 1] + [gB]
            env_ref = [R.build_env(dims, dims) for _ in range(numv - 1)]
            genv = [K.build_env(dims, dims, None, gpu_ctx) for _ in range(numv - 1)]
            o_ref = R.copy_mps(A)
            og = gA.clone()
            e_ref = R.build_env(dims, dims, wl)
            eg = K.build_env(dims, dims, wl, gpu_ctx)
            fn_ref = R.compress_sum_var_apply_H_right_ if right else R.compress_sum_var_apply_H_left_
            fn = K.compress_sum_var_apply_H_right_ if right else K.compress_sum_var_apply_H_left_
            fn_ref(o_ref, env_ref, e_ref, A, coef, terms_ref, H)
            fn(og, genv, eg, gA, coef, gterms, Hd)
            _sites_close(og, o_ref, 1e-10)


def test_compress_var_apply_H_full_sweeps(gpu_ctx):
    import mpsb200 as K
    na, chi = 9, 8
    A, dims = _random_lo(na, chi, 2, 21)
    p = OM.SpinChain(na, omega=0.5)
    jr_, _ = OM.jump_mpos(p)
    wl = [1] + [h.shape[2] for h in jr_]
    for sweeps in (1, 2):
        o_ref, e_ref = R.copy_mps(A), R.build_env(dims, dims, wl)
        R.compress_var_apply_H_(o_ref, e_ref, A, A, jr_, sweeps)
        gA = _mps(K, A, gpu_ctx)
        og, eg = gA.clone(), K.build_env(dims, dims, wl, gpu_ctx)
        K.compress_var_apply_H_(og, eg, gA, gA, K.MPO.from_sites(jr_, gpu_ctx), sweeps)
        _sites_close(og, o_ref, 1e-10)


def test_rk4_trajectory_step_matches_oracle_and_dense(gpu_ctx):
    """Full bond dimension: one RK4stp_apply_H_half! step equals the dense RK4 map."""
    import mpsb200 as K
    na, dt = 8, 0.01
    p = OM.SpinChain(na, omega=0.5)
    H = [OM.sm_hamiltonian(p, 1, dt / 2, 0), OM.sm_hamiltonian(p, 0, 1, dt / 2), OM.sm_hamiltonian(p, 1, dt / 2, dt)]
    Hd = [D.mpo_to_dense(h) for h in H]
    A, dims = R.mpsgroundstate(na, 16, 2)
    gA, _ = K.mpsgroundstate(na, 16, 2, gpu_ctx)
    gH = [K.MPO.from_sites(h, gpu_ctx) for h in H]
    g1, g2, g3, g0 = (gA.clone() for _ in range(4))
    ge = [K.build_env(dims, dims, None, gpu_ctx) for _ in range(3)]
    gop = K.build_env(dims, dims, [4] * (na + 1), gpu_ctx)
    A1, A2, A3, A0 = (R.copy_mps(A) for _ in range(4))
    e = [R.build_env(dims, dims) for _ in range(3)]
    eop = R.build_env(dims, dims, [4] * (na + 1))
    psi = D.mps_to_dense(A)
    for step in range(12):
        R.RK4stp_apply_H_half_(dt, H, A0, A, A1, A2, A3, *e, eop)
        K.RK4stp_apply_H_half_(dt, gH, g0, gA, g1, g2, g3, *ge, gop)
        psi = D.rk4_dense_step(*Hd, psi, dt)
        got = D.mps_to_dense(g0.sites())
        # the state itself (gauge invariant); raw sites may differ by the gauge of zero-weight
        # columns at exactly rank-deficient bonds (signed zeros decide a Householder sign there)
        assert np.abs(got - psi).max() < 1e-12
        assert np.abs(D.mps_to_dense(A0) - psi).max() < 1e-12
        A = R.copy_mps(A0)
        gA.copy_from(g0)


def test_rk4_density_inplace_matches_oracle(gpu_ctx):
    """10-argument in-place form on a vectorised rho (d=4, w=8), truncated bond dim."""
    import mpsb200 as K
    from mpsb200 import drivers as GDR, models as GM
    na, chi, dt, nsteps = 8, 16, 0.005, 20
    po = OM.SpinChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    pg = GM.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    rho_ref, obs_ref = ODR.run_density(po, chi, dt, nsteps, w=8, measure_int=5, pairs=((1, 2), (3, 6)))
    with perturbed_oracle_qr(1e-15):
        _, obs_pert = ODR.run_density(po, chi, dt, nsteps, w=8, measure_int=5, pairs=((1, 2), (3, 6)))
    b, obs = GDR.run_density(pg, chi, dt, nsteps, w=8, measure_int=5, pairs=((0, 1), (2, 5)), ctx=gpu_ctx)
    # chi=16 < 4^4 truncates; rho amplifies rounding faster than a pure state, so the gate is the
    # oracle's own spread under 1e-15 perturbations of its QR inputs (x100), and 1e-10 up to step 5
    for t, ((tr, see, spm), (tr_r, see_r, spm_r), (tr_p, see_p, spm_p)) in enumerate(zip(obs, obs_ref, obs_pert)):
        tol = 1e-10 if t <= 1 else 1e-10 + 100 * max(abs(tr_p - tr_r), np.abs(see_p - see_r).max(),
                                                     np.abs(spm_p - spm_r).max())
        assert abs(tr - tr_r) < tol
        assert np.abs(see - see_r).max() < tol
        assert np.abs(spm - spm_r).max() < tol
    assert 1 - fidelity(b.rho.sites(), rho_ref) < 1e-9


def test_observables_match_oracle(gpu_ctx):
    import mpsb200 as K
    A, dims = _random_lo(7, 8, 2, 31)
    B, _ = _random_lo(7, 8, 2, 32)
    gA, gB = _mps(K, A, gpu_ctx), _mps(K, B, gpu_ctx)
    assert abs(K.scal_prod(gA, gB) - R.scal_prod(A, B)) < 1e-12
    assert abs(K.scal_prod_no_conj(gA, gB) - R.scal_prod_no_conj(A, B)) < 1e-12
    p = OM.SpinChain(7, omega=0.3)
    jr_, _ = OM.jump_mpos(p)
    ir = R.applyMPOtoMPO(jr_, R.conj_mpo(jr_))
    assert abs(K.scal_op_prod(gA, K.MPO.from_sites(ir, gpu_ctx), gA) - R.scal_op_prod(A, ir, A)) < 1e-12
    e_ref = ODR.measure_excitations(A)
    assert np.abs(K.measure_local(gA, OM.hee) - e_ref).max() < 1e-13
    out = K.applyMPOtoMPS(gA, K.MPO.from_sites(jr_, gpu_ctx))
    _sites_close(out, R.applyMPOtoMPS(A, jr_), 1e-13)
    # norms, normalisation and the local-jump path
    C_ = R.copy_mps(A)
    C_[-1] = C_[-1] * 1.7
    gC = _mps(K, C_, gpu_ctx)
    assert abs(K.norm_lo(gC) - R.norm_lo(C_)) < 1e-12
    assert abs(K.normalize_lo_(gC) - R.normalize_lo_(C_)) < 1e-12
    _sites_close(gC, C_, 1e-14)
    K.apply_site_operator_(gC, 3, OM.hge)
    C_[2] = R.apply_site_operator_(C_[2], OM.hge)
    _sites_close(gC, C_, 1e-14)
    no_g = K.leftorthonormalizationQR_(gC)
    no_r = R.leftorthonormalizationQR_(C_)
    assert abs(no_g - no_r) < 1e-12
    _sites_close(gC, C_, 1e-10)


@pytest.mark.parametrize("order", [4, 1])
def test_trajectory_with_jumps_matches_oracle(gpu_ctx, order):
    """Quantum-jump loop (RK4 example, and with order=1 the first-order example whose coherent
    step is compress_var_apply_H! with 1 - i dt H): identical jump records for the same
    injected uniforms."""
    from mpsb200 import drivers as GDR, models as GM
    na, chi, dt, nsteps = 10, 16, 0.01, 60
    r1, r2 = ODR.uniforms(3, nsteps)
    r1 = np.where(np.arange(nsteps) % 7 == 6, 1.0, 0.0)       # force a jump every 7th step
    ref = ODR.run_trajectory(OM.SpinChain(na, omega=0.5), chi, dt, nsteps, r1, r2, measure_int=10, order=order)
    with perturbed_oracle_qr(1e-15):
        pert = ODR.run_trajectory(OM.SpinChain(na, omega=0.5), chi, dt, nsteps, r1, r2, measure_int=10, order=order)
    got = GDR.run_trajectory(GM.WaveguideChain(na, omega=0.5), chi, dt, nsteps, r1, r2, measure_int=10, ctx=gpu_ctx,
                             order=order)
    assert [j[:3] for j in got["jumps"]] == [j[:3] for j in ref["jumps"]]
    # r1 = 1 forces a jump only where p_coh < 1; the first-order step's p_coh can exceed 1
    assert len(ref["jumps"]) >= (5 if order == 4 else 3)
    # chi=16 < 2^5 truncates: the oracle itself moves by env under rounding-level perturbations of
    # its QR inputs; the GPU must stay within a small multiple of that envelope
    env_p = np.abs(pert["p_coh"] - ref["p_coh"]).max()
    env_e = np.abs(pert["e_pop"] - ref["e_pop"]).max()
    assert np.abs(got["p_coh"] - ref["p_coh"]).max() < 1e-12 + 100 * env_p
    assert np.abs(got["e_pop"] - ref["e_pop"]).max() < 1e-12 + 100 * env_e
    assert np.abs(got["p_coh"][:20] - ref["p_coh"][:20]).max() < 1e-12


def test_graph_replay_is_bitwise_eager(gpu_ctx):
    import mpsb200 as K
    from mpsb200 import drivers as GDR, models as GM
    p = GM.WaveguideChain(12, omega=0.5)
    outs = []
    for graphs in (False, True):
        gpu_ctx.set_graphs(graphs)
        b = GDR.TrajectoryBuffers(p, 16, 0.01, gpu_ctx)
        for _ in range(5):
            b.coherent_step()
            b.A.copy_from(b.A_coh)
        outs.append(np.concatenate([s.ravel() for s in b.A.sites()]))
    gpu_ctx.set_graphs(True)
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("graphs", [False, True])
def test_pipelined_rk4_is_bitwise_serial(gpu_ctx, graphs):
    """The two-stream RK4 step (each stage's environment initialisation beside the previous
    stage's sweep) computes exactly what the serial step computes, eagerly and replayed."""
    from mpsb200 import drivers as GDR, models as GM
    p = GM.WaveguideChain(10, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    outs = []
    gpu_ctx.set_graphs(graphs)
    for pipe in (False, True):
        gpu_ctx.set_pipeline(pipe)
        b = GDR.DensityBuffers(p, 32, 0.005, 8, gpu_ctx)
        for _ in range(6):
            b.step()
        outs.append(np.concatenate([s.ravel() for s in b.rho.sites()]))
    gpu_ctx.set_pipeline(True)
    gpu_ctx.set_graphs(True)
    assert np.array_equal(outs[0], outs[1])


def test_rk4_rho_chi512_blocked_qr(gpu_ctx):
    """The chi <= 512 configuration at reduced length (N=10, d=4, w=8): a random chi=64 state
    (mpsrandom semantics, normalised) expanded to chi=512; its 1024 x 512 and 2048 x 256 QRs
    take the blocked path inside expandmps and every sweep.  One 11-argument RK4 step against
    the oracle, through gauge-invariant quantities (the padded bonds are rank-deficient)."""
    import mpsb200 as K
    na, chi, dt = 10, 512, 0.005
    rng = np.random.default_rng(60)
    r64, _ = R.mpsrandom(na, 64, 4, rng)
    R.normalize_lo_(r64)
    rho, dims = R.expandmps(r64, chi)
    g, gdims = K.expandmps(K.MPS.from_sites(r64, gpu_ctx), chi)
    assert list(gdims) == list(dims)
    assert 1 - fidelity(g.sites(), rho) < 1e-12
    p = OM.SpinChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
    L = [OM.construct_L_spin_model(p, 1, dt / 2, 0, 8), OM.construct_L_spin_model(p, 0, 1, dt / 2, 8),
         OM.construct_L_spin_model(p, 1, dt / 2, dt, 8)]
    wl = [1] + [8] * (na - 1) + [1]
    def oracle_step():
        A0, A1, A2, A3 = (R.copy_mps(rho) for _ in range(4))
        e = [R.build_env(dims, dims) for _ in range(3)]
        R.RK4stp_apply_H_half_(dt, L, A0, rho, A1, A2, A3, *e, R.build_env(dims, dims, wl))
        return A0

    A0 = oracle_step()
    with perturbed_oracle_qr(1e-15):
        Ap = oracle_step()
    # the padded bonds make the projection subspaces depend on rounding-level details of the
    # junk columns: gate on the oracle's own spread under 1e-15 perturbations of its QR inputs
    env = 1 - fidelity(Ap, A0)
    g0, g1, g2, g3 = (g.clone() for _ in range(4))
    ge = [K.build_env(dims, dims, None, gpu_ctx) for _ in range(3)]
    K.RK4stp_apply_H_half_(dt, [K.MPO.from_sites(l, gpu_ctx) for l in L], g0, g, g1, g2, g3, *ge,
                           K.build_env(dims, dims, wl, gpu_ctx))
    got = g0.sites()
    assert abs(R.scal_prod(got, got) / R.scal_prod(A0, A0) - 1) < 1e-10
    assert 1 - fidelity(got, A0) < 1e-12 + 100 * env


@pytest.mark.parametrize("k", [3, 2])   # chimax 11 and 20
def test_trajectory_n64_log_uniform_chi(gpu_ctx, k):
    """The trajectory-ensemble configuration (N=64, d=2, w=4, dt=0.01, chimax_k = round(8*32^u_k),
    u_k ~ U[0,1) seeded by k), a few trajectories at reduced length: identical jump records and
    p_coh within the oracle's own rounding envelope."""
    from mpsb200 import drivers as GDR, models as GM
    na, dt, nsteps = 64, 0.01, 12
    chi = int(round(8 * 32 ** np.random.default_rng(k).random()))
    r1, r2 = ODR.uniforms(k, nsteps)
    r1 = np.where(np.arange(nsteps) % 5 == 4, 1.0, 0.0)       # a jump every 5th step
    ref = ODR.run_trajectory(OM.SpinChain(na, omega=0.5), chi, dt, nsteps, r1, r2, measure_int=4)
    with perturbed_oracle_qr(1e-15):
        pert = ODR.run_trajectory(OM.SpinChain(na, omega=0.5), chi, dt, nsteps, r1, r2, measure_int=4)
    got = GDR.run_trajectory(GM.WaveguideChain(na, omega=0.5), chi, dt, nsteps, r1, r2, measure_int=4, ctx=gpu_ctx)
    assert [j[:3] for j in got["jumps"]] == [j[:3] for j in ref["jumps"]]
    env_p = np.abs(pert["p_coh"] - ref["p_coh"]).max()
    assert np.abs(got["p_coh"] - ref["p_coh"]).max() < 1e-12 + 100 * env_p
    assert np.abs(got["e_pop"] - ref["e_pop"]).max() < 1e-12 + 100 * np.abs(pert["e_pop"] - ref["e_pop"]).max()
