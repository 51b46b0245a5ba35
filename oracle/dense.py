"""Exact dense references used to pin the restatement (TEST INFRASTRUCTURE ONLY).

With bond dimensions at their full value (dmax >= d^(na/2)) every single-site projection of
the sweeps is exact, so one ``RK4stp_apply_H_half_`` step must equal the dense RK4 map
psi -> -1/3 psi + 1/3 H1 psi + 2/3 psi2 + 1/3 H3 psi3 (src/timeevolution.jl:178-196), whose
algebra is the classic RK4 step psi + dt/6 (k1 + 2 k2 + 2 k3 + k4).
"""
import numpy as np

CT = np.complex128


def mps_to_dense(mps):
    """Contract an MPS to a vector indexed (s1, ..., sN), s1 slowest."""
    v = mps[0].reshape(mps[0].shape[1], mps[0].shape[2])
    for a in mps[1:]:
        v = np.einsum("xb,bsc->xsc", v, a).reshape(-1, a.shape[2])
    return v.reshape(-1)


def mpo_to_dense(mpo):
    """Contract an MPO O[wL, d_out, wR, d_in] to a matrix [(out...), (in...)]."""
    o = mpo[0]
    m = np.transpose(o[0], (0, 2, 1))  # (d_out, d_in, wR)
    for o in mpo[1:]:
        m = np.einsum("oiw,wpvj->opijv", m, o)
        do, di = m.shape[0] * m.shape[1], m.shape[2] * m.shape[3]
        m = m.reshape(do, di, -1)
    return m[:, :, 0]


def rk4_dense_step(H1, H2, H3, psi, dt):
    """The dense map that one RK4stp_apply_H_half! step computes at full bond dimension."""
    psi1 = H1 @ psi
    psi2 = psi + dt / 2 * (H2 @ psi1)
    psi3 = psi + dt * (H2 @ psi2)
    return -psi / 3 + psi1 / 3 + 2 * psi2 / 3 + (H3 @ psi3) / 3
