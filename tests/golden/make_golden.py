"""Regenerate the golden fixtures of this directory from the oracle.

    python tests/golden/make_golden.py

The reference (Julia 0.6) cannot run here, so the fixtures are the oracle's outputs on seeded
inputs; the oracle itself is pinned against dense exact evolution (tests/test_oracle.py).  For
the truncated long runs the fixture also stores the oracle's own spread under 1e-15 relative
perturbations of its QR inputs -- the envelope within which an independent implementation can
agree with it.  Inputs are rebuilt from the seeds by the builder functions below, which the
tests import.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import dense as D  # noqa: E402
from oracle import drivers as ODR  # noqa: E402
from oracle import models as OM  # noqa: E402
from oracle import mps_ref as R  # noqa: E402

CT = np.complex128
OP_SHAPE = (9, 2, 11, 3, 4, 7)   # chiL, d, chiR, wL, wR, chi0
TRAJ = dict(na=20, chi=32, dt=0.01, steps=200, seed=0, measure_int=10)   # the CPU-runnable configuration
RHO = dict(na=8, chi=16, dt=0.005, steps=40, w=8, measure_int=5, pairs=((1, 2), (3, 6)))
KIND = {"local": 0, "right": 1, "left": 2}


def crand(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(CT)


def op_inputs():
    """Seeded inputs of the op fixtures."""
    rng = np.random.default_rng(101)
    chiL, d, chiR, wL, wR, chi0 = OP_SHAPE
    return {"X": crand(rng, 64, 32),
            "A": crand(rng, chiL, d, chiR), "O": crand(rng, wL, d, wR, d),
            "Rr": crand(rng, chiR, wR, chi0), "L": crand(rng, chiL, wL, chi0),
            "A0r": crand(rng, chiL, d, chi0), "A0l": crand(rng, chi0, d, chiR)}


def padded_site():
    site = np.zeros((8, 4, 32), dtype=CT)
    site[0, :, 0] = [0.0, 1.0, 0.0, 0.0]
    return R.jr(site, 32, 32)


def make_ops():
    x = op_inputs()
    q, r = R.julia_qr(x["X"])
    aor = R.prod_AOR(x["A"], x["O"], x["Rr"])
    aol = R.prod_AOL(x["A"], x["O"], x["L"])
    return {"qr_Q": q, "qr_R": r, "qr_padded_Q": R.qrq(padded_site()),
            "prod_AOR": aor, "update_re": R.update_re(x["A0r"], aor),
            "prod_AOL": aol, "update_le": R.update_le(x["A0l"], aol)}


def traj_uniforms():
    return ODR.uniforms(TRAJ["seed"], TRAJ["steps"])


def run_traj():
    r1, r2 = traj_uniforms()
    rec = ODR.run_trajectory(OM.SpinChain(TRAJ["na"], omega=0.5), TRAJ["chi"], TRAJ["dt"], TRAJ["steps"], r1, r2,
                             measure_int=TRAJ["measure_int"])
    jumps = np.array([(j[0], KIND[j[1]], j[2]) for j in rec["jumps"]], dtype=np.int64).reshape(-1, 3)
    return rec["p_coh"], rec["e_pop"], jumps


def run_rho():
    p = OM.SpinChain(RHO["na"], gam_eg=0.1, omega=0.5, gam_phi=0.1)
    _, obs = ODR.run_density(p, RHO["chi"], RHO["dt"], RHO["steps"], w=RHO["w"], measure_int=RHO["measure_int"],
                             pairs=RHO["pairs"])
    return (np.array([o[0] for o in obs]), np.array([o[1] for o in obs]), np.array([o[2] for o in obs]))


def make_dense_pin():
    """Full bond dimension: 10 RK4 trajectory steps of N=6 equal the dense RK4 map."""
    na, dt = 6, 0.01
    p = OM.SpinChain(na, omega=0.5)
    H = [OM.sm_hamiltonian(p, 1, dt / 2, 0), OM.sm_hamiltonian(p, 0, 1, dt / 2), OM.sm_hamiltonian(p, 1, dt / 2, dt)]
    psi = D.mps_to_dense(R.mpsgroundstate(na, 8, 2)[0])
    for _ in range(10):
        psi = D.rk4_dense_step(*[D.mpo_to_dense(h) for h in H], psi, dt)
    return psi


def main():
    from gpu_util import perturbed_oracle_qr
    np.savez_compressed(os.path.join(HERE, "ops.npz"), **make_ops())
    p_coh, e_pop, jumps = run_traj()
    with perturbed_oracle_qr(1e-15):
        pp, pe, _ = run_traj()
    np.savez_compressed(os.path.join(HERE, "trajectory_n20_chi32.npz"), p_coh=p_coh, e_pop=e_pop, jumps=jumps,
                        env_p_coh=np.abs(pp - p_coh), env_e_pop=np.abs(pe - e_pop))
    tr, see, spm = run_rho()
    with perturbed_oracle_qr(1e-15):
        tp, sp, mp = run_rho()
    np.savez_compressed(os.path.join(HERE, "rho_n8_chi16.npz"), tr=tr, see=see, spm=spm,
                        env=np.maximum(np.abs(tp - tr), np.maximum(np.abs(sp - see).max(axis=1),
                                                                    np.abs(mp - spm).max(axis=1))))
    np.savez_compressed(os.path.join(HERE, "dense_rk4_n6.npz"), psi=make_dense_pin())


if __name__ == "__main__":
    main()
