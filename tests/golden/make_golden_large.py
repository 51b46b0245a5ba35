"""Golden fixtures at the benchmarked sizes, generated offline from the oracle.

    python tests/golden/make_golden_large.py rho40 [--perturbed]   # N=40, d=4, chi=128, w=8, 500 steps
    python tests/golden/make_golden_large.py rho60 [--perturbed]   # N=60, d=4, chi=512, w=8, random chi=64 start
    python tests/golden/make_golden_large.py traj64 [--perturbed]  # 8 trajectories, N=64, chi log-uniform 8..256
    python tests/golden/make_golden_large.py merge                 # combine the parts into the .npz fixtures

Each run writes one part file (``_parts/<name>[_pert].npz``, not committed); ``merge`` stores the
oracle's observables together with the envelope |oracle - oracle under 1e-15 relative
perturbations of its QR inputs|, the spread any independent implementation of the truncated
dynamics can be expected to stay within.  The oracle runs for hours at these sizes (a step of
the N=60, chi=512 density matrix is minutes on the host cores), which is why these fixtures are
separate from ``make_golden.py``.  Inputs are rebuilt from the parameters below by the tests.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import drivers as ODR  # noqa: E402
from oracle import models as OM  # noqa: E402
from oracle import mps_ref as R  # noqa: E402

PARTS = os.path.join(HERE, "_parts")
# the plain-FP64 density-matrix workload: waveguide Lindbladian with decay and dephasing
RHO40 = dict(na=40, chi=128, w=8, dt=0.005, steps=500, measure_int=10, gam_eg=0.1, omega=0.5, gam_phi=0.1,
             pairs=((1, 2), (10, 11), (20, 21), (5, 35)))
# the precision workload: same Lindbladian at N=60, chi=512, from a random chi=64 MPS
RHO60 = dict(na=60, chi=512, chi0=64, seed=60, w=8, dt=0.005, steps=3, measure_int=1, gam_eg=0.1, omega=0.5,
             gam_phi=0.1, pairs=((1, 2), (30, 31), (10, 50)))
# the batching workload, sampled: trajectories of the N=64 waveguide chain, per-trajectory chi
TRAJ64 = dict(na=64, dt=0.01, steps=30, measure_int=10, ntraj=8, chi_seed=3)
KIND = {"local": 0, "right": 1, "left": 2}


def traj64_chis():
    """chi_k = round(8 * 32**u_k), u_k ~ U[0,1) from a seeded generator, with the largest
    forced to 256 and the second largest to >= 128 so that the sample covers the top buckets."""
    u = np.random.default_rng(TRAJ64["chi_seed"]).random(TRAJ64["ntraj"])
    chis = [int(round(8 * 32 ** x)) for x in u]
    chis[int(np.argmax(chis))] = 256
    order = np.argsort(chis)
    if chis[int(order[-2])] < 128:
        chis[int(order[-2])] = 128
    return chis


def rho60_initial():
    """Random chi=64 MPS (complex Gaussian, seeded, left-orthogonal, unit norm) expanded to chi=512."""
    P = RHO60
    rng = np.random.default_rng(P["seed"])
    rho, _ = R.mpsrandom(P["na"], P["chi0"], 4, rng)
    R.normalize_lo_(rho)
    return R.expandmps(rho, P["chi"])[0]


def chain(P):
    return OM.SpinChain(P["na"], gam_eg=P["gam_eg"], omega=P["omega"], gam_phi=P["gam_phi"])


def _obs_dict(obs):
    return {"tr": np.array([o[0] for o in obs]), "see": np.array([o[1] for o in obs]),
            "spm": np.array([o[2] for o in obs])}


def run_rho40():
    P = RHO40
    t0 = time.time()
    _, obs = ODR.run_density(chain(P), P["chi"], P["dt"], P["steps"], w=P["w"], measure_int=P["measure_int"],
                             pairs=P["pairs"],
                             progress=lambda i: print("rho40 step", i, "%.0f s" % (time.time() - t0), flush=True))
    return _obs_dict(obs)


def run_rho60():
    P = RHO60
    t0 = time.time()
    rho = rho60_initial()
    print("rho60 initial state %.0f s" % (time.time() - t0), flush=True)
    _, obs = ODR.run_density(chain(P), P["chi"], P["dt"], P["steps"], w=P["w"], measure_int=P["measure_int"],
                             pairs=P["pairs"], rho=rho,
                             progress=lambda i: print("rho60 step", i, "%.0f s" % (time.time() - t0), flush=True))
    return _obs_dict(obs)


def run_traj64():
    P = TRAJ64
    out = {"chis": np.array(traj64_chis())}
    for k, chi in enumerate(out["chis"]):
        t0 = time.time()
        r1, r2 = ODR.uniforms(k, P["steps"])
        rec = ODR.run_trajectory(OM.SpinChain(P["na"], omega=0.5), int(chi), P["dt"], P["steps"], r1, r2,
                                 measure_int=P["measure_int"])
        jumps = np.array([(j[0], KIND[j[1]], j[2]) for j in rec["jumps"]], dtype=np.int64).reshape(-1, 3)
        out["p_coh_%d" % k] = rec["p_coh"]
        out["e_pop_%d" % k] = rec["e_pop"]
        out["jumps_%d" % k] = jumps
        print("traj64 k=%d chi=%d jumps=%d %.0f s" % (k, chi, len(jumps), time.time() - t0), flush=True)
    return out


def _rho_env(a, b):
    return np.maximum(np.abs(b["tr"] - a["tr"]), np.maximum(np.abs(b["see"] - a["see"]).max(axis=1),
                                                            np.abs(b["spm"] - a["spm"]).max(axis=1)))


def merge():
    def load(name):
        a = dict(np.load(os.path.join(PARTS, name + ".npz")))
        b = dict(np.load(os.path.join(PARTS, name + "_pert.npz")))
        return a, b

    for name, out in (("rho40", "rho_n40_chi128.npz"), ("rho60", "rho_n60_chi512.npz")):
        if os.path.exists(os.path.join(PARTS, name + "_pert.npz")):
            a, b = load(name)
            np.savez_compressed(os.path.join(HERE, out), env=_rho_env(a, b), **a)
    if os.path.exists(os.path.join(PARTS, "traj64_pert.npz")):
        a, b = load("traj64")
        extra = {}
        for k in range(len(a["chis"])):
            extra["env_p_coh_%d" % k] = np.abs(b["p_coh_%d" % k] - a["p_coh_%d" % k])
            extra["env_e_pop_%d" % k] = np.abs(b["e_pop_%d" % k] - a["e_pop_%d" % k])
        np.savez_compressed(os.path.join(HERE, "traj_n64_batch8.npz"), **a, **extra)


def main():
    which = sys.argv[1]
    if which == "merge":
        merge()
        return
    pert = "--perturbed" in sys.argv
    fn = {"rho40": run_rho40, "rho60": run_rho60, "traj64": run_traj64}[which]
    os.makedirs(PARTS, exist_ok=True)
    if pert:
        from gpu_util import perturbed_oracle_qr
        with perturbed_oracle_qr(1e-15):
            res = fn()
    else:
        res = fn()
    np.savez_compressed(os.path.join(PARTS, which + ("_pert" if pert else "") + ".npz"), **res)


if __name__ == "__main__":
    main()
