"""Time loops of the reference examples, restated on the oracle (TEST INFRASTRUCTURE ONLY).

* ``run_trajectory``  examples/spin_model_quantum_trajectory_rk4.jl:44-217 (coherent RK4
  step, jump probabilities from compressed jump MPOs, jump selection, measurements); with
  order=1, examples/spin_model_quantum_trajectory.jl:42-190 (coherent step
  compress_var_apply_H!(A_coh, envop, A, A, expH, 1) with expH = 1 - i dt H)
* ``run_density``     examples/spin_model_density_matrix.jl:36-203 (in-place RK4 of vec(rho),
  trace / population measurements)

Julia's ``srand(setrand); r1 = rand(tstep); r2 = rand(tstep)`` stream cannot be reproduced
without Julia, so the uniforms ``r1``/``r2`` are injected by the caller and the same arrays
are fed to the GPU engine.
"""
import numpy as np

from . import mps_ref as R
from . import models as M


def measure_excitations(A, op=None):
    """examples/spin_model_quantum_trajectory_rk4.jl:220-231: local <op_n> of a left-normalised MPS."""
    op = M.hee if op is None else op
    na = len(A)
    out = np.zeros(na)
    env = np.ones((1, 1), dtype=R.CT)
    for n in range(na - 1, -1, -1):
        Aenv = R.prod_LR(A[n], env)
        out[n] = float(np.real(R.local_exp(Aenv, A[n], op)))
        env = R.update_renv(A[n], Aenv)
    return out


def uniforms(seed, nsteps):
    """The injected stand-in for Julia's r1, r2 draws (NumPy PCG64, documented seed)."""
    g = np.random.default_rng(seed)
    return g.random(nsteps), g.random(nsteps)


def run_trajectory(p, dmax, dt, nsteps, r1, r2, measure_int=10, order=4):
    """One quantum trajectory; returns a dict of records (jumps, p_coh, e_pop, I_r, final MPS)."""
    na = p.na
    A, dims = R.mpsgroundstate(na, dmax, 2)
    jumpright, jumpleft = M.jump_mpos(p, 0.0)
    ir_mpo = R.applyMPOtoMPO(jumpright, R.conj_mpo(jumpright))
    envop = R.build_env(dims, dims, [4] * (na + 1))
    envop_jump = R.build_env(dims, dims, [2] * (na + 1))
    env1, env2, env3 = (R.build_env(dims, dims) for _ in range(3))
    A_coh, A_r, A_l, A1, A2, A3 = (R.copy_mps(A) for _ in range(6))
    t = np.arange(nsteps + 1) * dt
    H1 = M.sm_hamiltonian(p, 1, dt / 2, t[0])
    H2 = M.sm_hamiltonian(p, 0, 1, t[0] + dt / 2)
    H3 = M.sm_hamiltonian(p, 1, dt / 2, t[1])
    H = [H1, H2, H3]
    expH = M.sm_hamiltonian(p, 1, dt, t[0])
    rec = {"p_coh": np.zeros(nsteps), "jumps": [], "e_pop": [M_measure(A)],
           "I_r": [R.scal_op_prod(A, ir_mpo, A)], "dims": dims}
    for i in range(nsteps):
        if order == 1:
            M.update_h(expH, p, 1, dt, t[i])
            R.compress_var_apply_H_(A_coh, envop, A, A, expH, 1)
        else:
            M.update_h(H1, p, 1, dt / 2, t[i])
            M.update_h(H2, p, 0, 1, t[i] + dt / 2)
            M.update_h(H3, p, 1, dt / 2, t[i + 1])
            R.RK4stp_apply_H_half_(dt, H, A_coh, A, A1, A2, A3, env1, env2, env3, envop)
        p_coh = R.normalize_lo_(A_coh)
        rec["p_coh"][i] = p_coh
        if r1[i] < p_coh:
            A = R.copy_mps(A_coh)
        else:
            jumpright[0][0, :, 1, :] = p.f(t[i]) * M.id2 + 1j * np.sqrt(p.gam_1d[0] / 2) * np.exp(-1j * p.k_wg * p.rj[0]) * M.hge
            R.compress_var_apply_H_(A_r, envop_jump, A, A, jumpright, 1)
            p_r = R.normalize_lo_(A_r)
            R.compress_var_apply_H_(A_l, envop_jump, A, A, jumpleft, 1)
            p_l = R.normalize_lo_(A_l)
            epop = measure_excitations(A)
            p_acc = np.zeros(na + 3)
            for j in range(na):
                p_acc[j + 1] = p_acc[j] + dt * p.gam_eg * epop[j]
            p_acc[na + 1] = p_acc[na] + dt * p_r
            p_acc[na + 2] = p_acc[na + 1] + dt * p_l
            p_sum = p_acc[-1]
            p_acc = p_acc / p_acc[-1]
            if r2[i] < p_acc[na]:
                for j in range(na):
                    if r2[i] < p_acc[j + 1]:
                        A[j] = R.apply_site_operator_(A[j], M.hge)
                        R.leftorthonormalizationQR_(A)
                        rec["jumps"].append((i, "local", j + 1, p_coh, p_sum))
                        break
            elif r2[i] < p_acc[na + 1]:
                A = R.copy_mps(A_r)
                rec["jumps"].append((i, "right", 0, p_coh, p_sum))
            else:
                A = R.copy_mps(A_l)
                rec["jumps"].append((i, "left", 0, p_coh, p_sum))
        if (i + 1) % measure_int == 0:
            rec["e_pop"].append(M_measure(A))
            rec["I_r"].append(R.scal_op_prod(A, ir_mpo, A))
    rec["A"] = A
    rec["e_pop"] = np.array(rec["e_pop"])
    rec["I_r"] = np.array(rec["I_r"])
    return rec


def M_measure(A):
    return measure_excitations(A)


def rho_observables(rho, pairs=((1, 2),)):
    """Tr rho, <sigma_ee_i> for every site and <sigma+_i sigma-_j> for ``pairs`` (1-based)."""
    na = len(rho)
    tr = R.scal_prod_no_conj(M.identity_lmps(na), rho)
    see = np.array([R.scal_prod_no_conj(M.rho_site_functional_lmps(na, {j: M.SEE_VEC}), rho)
                    for j in range(1, na + 1)])
    spm = np.array([R.scal_prod_no_conj(M.rho_site_functional_lmps(na, {i: M.SP_VEC, j: M.SM_VEC}), rho)
                    for (i, j) in pairs])
    return tr, see, spm


def run_density(p, dmax, dt, nsteps, w=6, measure_int=10, pairs=((1, 2),), rho=None, progress=None):
    """In-place density-matrix RK4 (the 10-argument form) from the all-down product state
    (or from ``rho``); ``progress(i)``, when given, is called after every step."""
    na = p.na
    if rho is None:
        rho, dims = R.mpsgroundstate(na, dmax, 4)
    else:
        dims = [1] + [a.shape[2] for a in rho]
    rho1, rho2, rho3 = (R.copy_mps(rho) for _ in range(3))
    env1, env2, env3 = (R.build_env(dims, dims) for _ in range(3))
    envop = R.build_env(dims, dims, [w] * (na + 1))
    t = np.arange(nsteps + 1) * dt
    L = [construct(p, 1, dt / 2, t[0], w), construct(p, 0, 1, t[0] + dt / 2, w), construct(p, 1, dt / 2, t[1], w)]
    obs = [rho_observables(rho, pairs)]
    for i in range(nsteps):
        R.RK4stp_apply_H_half_(dt, L, rho, rho, rho1, rho2, rho3, env1, env2, env3, envop)
        if (i + 1) % measure_int == 0:
            obs.append(rho_observables(rho, pairs))
        if progress is not None:
            progress(i + 1)
    return rho, obs


def construct(p, con, delt, time, w):
    return M.construct_L_spin_model(p, con, delt, time, w=w)
