"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the oracle): the
oracle must keep reproducing them, and the GPU path must match them -- bit for bit where the
arithmetic is short, within the stored rounding envelope for the long truncated runs."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

from oracle import dense as D  # noqa: E402
from oracle import mps_ref as R  # noqa: E402


def _load(name):
    return np.load(os.path.join(HERE, "golden", name))


def test_oracle_reproduces_op_fixtures():
    want = _load("ops.npz")
    got = G.make_ops()
    for k in want.files:
        assert np.abs(got[k] - want[k]).max() <= 1e-13 * max(1.0, np.abs(want[k]).max()), k


def test_oracle_reproduces_trajectory_fixture():
    f = _load("trajectory_n20_chi32.npz")
    p_coh, e_pop, jumps = G.run_traj()
    assert np.array_equal(jumps, f["jumps"]) and len(jumps) > 0
    assert np.all(np.abs(p_coh - f["p_coh"]) <= 1e-13 + 10 * f["env_p_coh"].max())
    assert np.all(np.abs(e_pop - f["e_pop"]) <= 1e-13 + 10 * f["env_e_pop"].max())


def test_oracle_reproduces_rho_fixture():
    f = _load("rho_n8_chi16.npz")
    tr, see, spm = G.run_rho()
    tol = 1e-12 + 10 * f["env"][:, None]
    assert np.all(np.abs(see - f["see"]) <= tol) and np.all(np.abs(spm - f["spm"]) <= tol)
    assert np.all(np.abs(tr - f["tr"]) <= tol[:, 0])


def test_dense_pin_matches_oracle_full_bond_rk4():
    from oracle import models as OM
    na, dt = 6, 0.01
    p = OM.SpinChain(na, omega=0.5)
    H = [OM.sm_hamiltonian(p, 1, dt / 2, 0), OM.sm_hamiltonian(p, 0, 1, dt / 2), OM.sm_hamiltonian(p, 1, dt / 2, dt)]
    A, dims = R.mpsgroundstate(na, 8, 2)
    A1, A2, A3, A0 = (R.copy_mps(A) for _ in range(4))
    e = [R.build_env(dims, dims) for _ in range(3)]
    eop = R.build_env(dims, dims, [4] * (na + 1))
    for _ in range(10):
        R.RK4stp_apply_H_half_(dt, H, A0, A, A1, A2, A3, *e, eop)
        A = R.copy_mps(A0)
    assert np.abs(D.mps_to_dense(A) - _load("dense_rk4_n6.npz")["psi"]).max() < 1e-13


# ---------------------------------------------------------------- the GPU against the fixtures
@pytest.mark.gpu
def test_gpu_ops_match_fixtures(gpu_ctx):
    import torch
    from gpu_util import empty_dev, from_dev, to_dev
    from mpsb200 import _lib
    f, x = _load("ops.npz"), G.op_inputs()
    p = lambda t: C.c_void_p(t.data_ptr())   # noqa: E731

    def call(name, *args):
        torch.cuda.synchronize()
        _lib.call(name, gpu_ctx.h, *args)
        gpu_ctx.sync()

    dX, dQ, dR = to_dev(x["X"]), empty_dev((64, 32)), empty_dev((32, 32))
    call("mpsb_op_qr", p(dX), p(dQ), p(dR), 64, 32)
    assert np.abs(from_dev(dQ, (64, 32)) - f["qr_Q"]).max() < 1e-12
    assert np.abs(from_dev(dR, (32, 32)) - f["qr_R"]).max() < 1e-12 * np.abs(f["qr_R"]).max()
    dP = to_dev(G.padded_site())
    call("mpsb_op_qr", p(dP), p(dP), None, 32, 32)
    assert np.abs(from_dev(dP, (32, 32)) - f["qr_padded_Q"]).max() < 1e-15
    chiL, d, chiR, wL, wR, chi0 = G.OP_SHAPE
    dA, dO, dRr, dL = to_dev(x["A"]), to_dev(x["O"]), to_dev(x["Rr"]), to_dev(x["L"])

    def close(dev, key):
        want = f[key]
        return np.abs(from_dev(dev, want.shape) - want).max() < 1e-12 * np.abs(want).max()

    dAOR, dAOL = empty_dev(f["prod_AOR"].shape), empty_dev(f["prod_AOL"].shape)
    call("mpsb_op_prod_AOR", p(dA), p(dO), p(dRr), p(dAOR), chiL, d, chiR, wL, wR, chi0)
    assert close(dAOR, "prod_AOR")
    call("mpsb_op_prod_AOL", p(dA), p(dO), p(dL), p(dAOL), chiL, d, chiR, wL, wR, chi0)
    assert close(dAOL, "prod_AOL")
    denv = empty_dev(f["update_re"].shape)
    call("mpsb_op_update_re", p(to_dev(x["A0r"])), p(dAOR), p(denv), chiL, wL, d, chi0, chiL)
    assert close(denv, "update_re")
    denv = empty_dev(f["update_le"].shape)
    call("mpsb_op_update_le", p(to_dev(x["A0l"])), p(dAOL), p(denv), chi0, d, chiR, wR, chiR)
    assert close(denv, "update_le")


@pytest.mark.gpu
def test_gpu_trajectory_matches_fixture(gpu_ctx):
    """The CPU-runnable configuration in full: N=20, chi=32, dt=0.01, 200 steps, seed 0."""
    from mpsb200 import drivers as GDR, models as GM
    f = _load("trajectory_n20_chi32.npz")
    T = G.TRAJ
    r1, r2 = G.traj_uniforms()
    rec = GDR.run_trajectory(GM.WaveguideChain(T["na"], omega=0.5), T["chi"], T["dt"], T["steps"], r1, r2,
                             measure_int=T["measure_int"], ctx=gpu_ctx)
    jumps = np.array([(j[0], G.KIND[j[1]], j[2]) for j in rec["jumps"]], dtype=np.int64).reshape(-1, 3)
    assert np.array_equal(jumps, f["jumps"])
    assert np.all(np.abs(rec["p_coh"] - f["p_coh"]) <= 1e-12 + 100 * f["env_p_coh"].max())
    assert np.all(np.abs(rec["e_pop"] - f["e_pop"]) <= 1e-12 + 100 * f["env_e_pop"].max())
    assert np.abs(rec["p_coh"][:20] - f["p_coh"][:20]).max() < 1e-12


@pytest.mark.gpu
def test_gpu_rho_matches_fixture(gpu_ctx):
    from mpsb200 import drivers as GDR, models as GM
    f = _load("rho_n8_chi16.npz")
    Rh = G.RHO
    pairs = tuple((i - 1, j - 1) for i, j in Rh["pairs"])   # the fixture's pairs are 1-based
    _, obs = GDR.run_density(GM.WaveguideChain(Rh["na"], gam_eg=0.1, omega=0.5, gam_phi=0.1), Rh["chi"], Rh["dt"],
                             Rh["steps"], w=Rh["w"], measure_int=Rh["measure_int"], pairs=pairs, ctx=gpu_ctx)
    for t, (tr, see, spm) in enumerate(obs):
        tol = 1e-10 + 100 * f["env"][t]
        assert abs(tr - f["tr"][t]) < tol
        assert np.abs(see - f["see"][t]).max() < tol and np.abs(spm - f["spm"][t]).max() < tol


@pytest.mark.gpu
def test_gpu_full_bond_rk4_matches_dense_pin(gpu_ctx):
    import mpsb200 as K
    from oracle import models as OM
    na, dt = 6, 0.01
    p = OM.SpinChain(na, omega=0.5)
    H = [K.MPO.from_sites(h, gpu_ctx) for h in
         (OM.sm_hamiltonian(p, 1, dt / 2, 0), OM.sm_hamiltonian(p, 0, 1, dt / 2), OM.sm_hamiltonian(p, 1, dt / 2, dt))]
    A, dims = K.mpsgroundstate(na, 8, 2, gpu_ctx)
    g0, g1, g2, g3 = (A.clone() for _ in range(4))
    e = [K.build_env(dims, dims, None, gpu_ctx) for _ in range(3)]
    eop = K.build_env(dims, dims, [4] * (na + 1), gpu_ctx)
    for _ in range(10):
        K.RK4stp_apply_H_half_(dt, H, g0, A, g1, g2, g3, *e, eop)
        A.copy_from(g0)
    assert np.abs(D.mps_to_dense(g0.sites()) - _load("dense_rk4_n6.npz")["psi"]).max() < 1e-12
