"""The reference examples' time loops on the GPU engine.

* ``run_trajectory``  examples/spin_model_quantum_trajectory_rk4.jl:44-217; with order=1
  examples/spin_model_quantum_trajectory.jl:42-190 (first-order coherent step)
* ``run_density``     examples/spin_model_density_matrix.jl:36-203 (10-argument in-place RK4)

Every tensor operation is a libmpsb200 call; the host only makes the jump decisions from the
FP64 probabilities the device returns (``r1``/``r2`` uniforms are injected by the caller, the
stand-in for Julia's ``srand(setrand); rand(tstep)`` stream).
"""
import os

import numpy as np

from . import core as K
from . import models as Mo


class TrajectoryBuffers:
    """Device-resident state of one trajectory (the example's A, A_coh, A_r, A_l, A1..A3, envs)."""

    def __init__(self, p, dmax, dt, ctx=None, order=4):
        self.p, self.dt, self.order = p, dt, order
        na = p.na
        self.A, self.dims = K.mpsgroundstate(na, dmax, 2, ctx)
        ctx = self.A.ctx
        self.ctx = ctx
        dims = self.dims
        self.A_coh, self.A_r, self.A_l, self.A1, self.A2, self.A3 = (self.A.clone() for _ in range(6))
        self.envop = K.build_env(dims, dims, [4] * (na + 1), ctx)
        self.envop_jump = K.build_env(dims, dims, [2] * (na + 1), ctx)
        self.env1, self.env2, self.env3 = (K.build_env(dims, dims, None, ctx) for _ in range(3))
        self.H = [K.MPO.from_sites(Mo.sm_hamiltonian(p, 1, dt / 2, 0.0), ctx),
                  K.MPO.from_sites(Mo.sm_hamiltonian(p, 0, 1, dt / 2), ctx),
                  K.MPO.from_sites(Mo.sm_hamiltonian(p, 1, dt / 2, dt), ctx)]
        self.expH = K.MPO.from_sites(Mo.sm_hamiltonian(p, 1, dt, 0.0), ctx) if order == 1 else None
        jr_, jl_ = Mo.jump_mpos(p, 0.0)
        self.jumpright = K.MPO.from_sites(jr_, ctx)
        self.jumpleft = K.MPO.from_sites(jl_, ctx)

    def coherent_step(self):
        if self.order == 1:   # compress_var_apply_H!(A_coh, envop, A, A, expH, 1)
            K.compress_var_apply_H_(self.A_coh, self.envop, self.A, self.A, self.expH, 1)
        else:
            K.RK4stp_apply_H_half_(self.dt, self.H, self.A_coh, self.A, self.A1, self.A2, self.A3,
                                   self.env1, self.env2, self.env3, self.envop)
        return K.normalize_lo_(self.A_coh)


def trajectory_decision(b, i, p_coh, r1, r2, rec):
    """The jump branch of step i (examples/spin_model_quantum_trajectory_rk4.jl:105-190): keep
    the coherent state when r1[i] < p_coh, else pick a local decay or a waveguide jump from the
    accumulated probabilities with r2[i] and apply it; jumps are appended to rec["jumps"]."""
    p, dt, na = b.p, b.dt, b.p.na
    if r1[i] < p_coh:
        b.A.copy_from(b.A_coh)
        return
    K.compress_var_apply_H_(b.A_r, b.envop_jump, b.A, b.A, b.jumpright, 1)
    p_r = K.normalize_lo_(b.A_r)
    K.compress_var_apply_H_(b.A_l, b.envop_jump, b.A, b.A, b.jumpleft, 1)
    p_l = K.normalize_lo_(b.A_l)
    epop = K.measure_local(b.A, Mo.E_E)
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
                K.apply_site_operator_(b.A, j + 1, Mo.SM)
                K.leftorthonormalizationQR_(b.A)
                rec["jumps"].append((i, "local", j + 1, p_coh, p_sum))
                break
    elif r2[i] < p_acc[na + 1]:
        b.A.copy_from(b.A_r)
        rec["jumps"].append((i, "right", 0, p_coh, p_sum))
    else:
        b.A.copy_from(b.A_l)
        rec["jumps"].append((i, "left", 0, p_coh, p_sum))


def run_trajectory(p, dmax, dt, nsteps, r1, r2, measure_int=10, ctx=None, order=4):
    b = TrajectoryBuffers(p, dmax, dt, ctx, order)
    rec = {"p_coh": np.zeros(nsteps), "jumps": [], "e_pop": [K.measure_local(b.A, Mo.E_E)]}
    for i in range(nsteps):
        p_coh = b.coherent_step()
        rec["p_coh"][i] = p_coh
        trajectory_decision(b, i, p_coh, r1, r2, rec)
        if (i + 1) % measure_int == 0:
            rec["e_pop"].append(K.measure_local(b.A, Mo.E_E))
    rec["e_pop"] = np.array(rec["e_pop"])
    rec["buffers"] = b
    return rec


class DensityBuffers:
    """Device-resident state of one density-matrix evolution (rho, rho1..3, envs, L MPOs)."""

    def __init__(self, p, dmax, dt, w=6, ctx=None, rho=None):
        na = p.na
        if rho is None:
            self.rho, self.dims = K.mpsgroundstate(na, dmax, 4, ctx)
        else:
            self.rho, self.dims = rho, list(rho.dims)
        ctx = self.rho.ctx
        self.ctx, self.dt, self.p, self.w = ctx, dt, p, w
        dims = self.dims
        self.rho1, self.rho2, self.rho3 = (self.rho.clone() for _ in range(3))
        self.env1, self.env2, self.env3 = (K.build_env(dims, dims, None, ctx) for _ in range(3))
        self.envop = K.build_env(dims, dims, [max(6, w)] * (na + 1), ctx)
        self.L = [K.MPO.from_sites(Mo.construct_L_spin_model(p, 1, dt / 2, 0.0, w), ctx),
                  K.MPO.from_sites(Mo.construct_L_spin_model(p, 0, 1, dt / 2, w), ctx),
                  K.MPO.from_sites(Mo.construct_L_spin_model(p, 1, dt / 2, dt, w), ctx)]
        self.trace_fn = K.MPS.from_sites(Mo.functional_sites(na, {}), ctx)
        self._see = [K.MPS.from_sites(Mo.functional_sites(na, {j: Mo.SEE_VEC}), ctx) for j in range(na)]

    def step(self):
        K.RK4stp_apply_H_half_(self.dt, self.L, self.rho, self.rho1, self.rho2, self.rho3,
                               self.env1, self.env2, self.env3, self.envop)

    def observables(self, pairs=((0, 1),)):
        tr = K.scal_prod_no_conj(self.trace_fn, self.rho)
        see = np.array([K.scal_prod_no_conj(f, self.rho) for f in self._see])
        spm = []
        for (i, j) in pairs:
            f = K.MPS.from_sites(Mo.functional_sites(self.p.na, {i: Mo.SP_VEC, j: Mo.SM_VEC}), self.ctx)
            spm.append(K.scal_prod_no_conj(f, self.rho))
        return tr, see, np.array(spm)


def run_density(p, dmax, dt, nsteps, w=6, measure_int=10, pairs=((0, 1),), ctx=None, rho=None,
                checkpoint=None, checkpoint_int=0):
    """The density-matrix time loop (examples/spin_model_density_matrix.jl): nsteps in-place RK4
    steps with (Tr rho, <see_i>, <s+_i s-_j>) every measure_int steps.

    With `checkpoint` (a file path) the run restarts from that file when it exists -- rho and
    the step index i_last, as the reference's restart example reads them -- and rewrites it
    every `checkpoint_int` steps (0: only at the end)."""
    from . import checkpoint as CK
    i0, obs = 0, None
    if checkpoint and os.path.exists(checkpoint):
        st = CK.read_data_file(checkpoint, ctx)
        if abs(float(st["dt"]) - dt) > 0 or int(st["d_max"]) != dmax or int(st["measure_int"]) != measure_int:
            raise ValueError("checkpoint %s was written with other dt / d_max / measure_int" % checkpoint)
        rho, i0 = st["rho"], int(st["i_last"])
        obs = [(t, s_, m_) for t, s_, m_ in zip(st["tr_rho"], st["see"], st["spm"])]
    b = DensityBuffers(p, dmax, dt, w, ctx, rho)
    if obs is None:
        obs = [b.observables(pairs)]

    def save(i):
        CK.write_data_file(checkpoint, {
            "rho": b.rho, "i_last": i, "dt": dt, "d_max": dmax, "measure_int": measure_int, "na": p.na,
            "tr_rho": np.array([o[0] for o in obs]), "see": np.array([o[1] for o in obs]),
            "spm": np.array([o[2] for o in obs])})

    for i in range(i0, nsteps):
        b.step()
        if (i + 1) % measure_int == 0:
            obs.append(b.observables(pairs))
        if checkpoint and checkpoint_int and (i + 1) % checkpoint_int == 0 and i + 1 < nsteps:
            save(i + 1)
    if checkpoint:
        save(nsteps)
    return b, obs
