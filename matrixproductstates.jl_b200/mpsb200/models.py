"""Waveguide spin-model generators used by the examples of the reference (host-side MPO data).

* ``sm_hamiltonian``         examples/spin_model_quantum_trajectory_rk4.jl:235-293 (w=4, d=2)
* ``jump_mpos``              examples/spin_model_quantum_trajectory_rk4.jl:51-55   (w=2)
* ``construct_L_spin_model`` examples/spin_model_density_matrix.jl:245-317          (w=6, d=4)

Both generators add two local terms named by the benchmark workloads, zero by default:
``omega`` (Hermitian drive -omega(sigma+ + sigma-)) and ``gam_phi`` (pure dephasing with
Lindblad operator sqrt(gam_phi) sigma_ee).  ``w > 6`` pads the Lindbladian MPO with zero
channels (kept before the closing channel) to reach a requested bond width.
Site basis [g, e]; vectorised rho basis [gg, ge, eg, ee] with kron(X, Y) vec(rho) = vec(X rho Y^T).
"""
import numpy as np

CT = np.complex128
G_G = np.array([[1, 0], [0, 0]], dtype=CT)
E_E = np.array([[0, 0], [0, 1]], dtype=CT)
SM = np.array([[0, 1], [0, 0]], dtype=CT)     # hge = |g><e| = sigma-
SP = SM.T.copy()                              # heg = sigma+
I2 = np.eye(2, dtype=CT)


class WaveguideChain:
    def __init__(self, na, gam_1d=1.0, gam_eg=0.0, del_p=0.0, k_wg=0.5 * np.pi, rj=None,
                 k_in=0.5 * np.pi, f=None, omega=0.0, gam_phi=0.0):
        self.na = int(na)
        self.gam_1d = np.full(self.na, float(gam_1d)) if np.isscalar(gam_1d) else np.asarray(gam_1d, float)
        self.gam_eg, self.del_p, self.k_wg = float(gam_eg), float(del_p), float(k_wg)
        self.rj = np.arange(1.0, self.na + 1.0) if rj is None else np.asarray(rj, float)
        self.k_in = float(k_in)
        self.f = f or (lambda t: 0.0)
        self.omega, self.gam_phi = float(omega), float(gam_phi)


def _local_h(p, j, con, delt, t):
    g, ft = p.gam_1d[j], p.f(t)
    return con * I2 / p.na + delt * ((1j * p.del_p - (p.gam_eg + g) / 2) * E_E
                                     + 1j * np.sqrt(g / 2) * ft * np.exp(1j * p.k_in * p.rj[j]) * SP
                                     - abs(ft) ** 2 / (2 * p.na) * I2 + 1j * p.omega * (SP + SM))


def sm_hamiltonian(p, con, delt, t):
    """MPO of con*1 + delt*(-i H_eff): list of O[wL, 2, wR, 2] site tensors."""
    na = p.na
    ph = np.exp(1j * p.k_wg * np.diff(p.rj))
    cp = np.sqrt(delt * p.gam_1d / 2)
    out = []
    for j in range(na):
        o = np.zeros((4, 2, 4, 2), dtype=CT)
        if j < na - 1:
            o[0, :, 0, :] = I2
            o[0, :, 1, :] = -cp[j] * ph[j] * SP
            o[0, :, 2, :] = -cp[j] * ph[j] * SM
            o[1, :, 1, :] = ph[j] * I2
            o[2, :, 2, :] = ph[j] * I2
        o[0, :, 3, :] = _local_h(p, j, con, delt, t)
        o[1, :, 3, :] = cp[j] * SM
        o[2, :, 3, :] = cp[j] * SP
        o[3, :, 3, :] = I2
        if j == 0:
            o = o[0:1]
        if j == na - 1:
            o = o[:, :, 3:4]
        out.append(np.ascontiguousarray(o))
    return out


def jump_mpos(p, t=0.0):
    """(jumpright, jumpleft): sum_j i sqrt(gam/2) e^{-/+ i k r_j} sigma-_j as w=2 MPOs."""
    out = []
    for sgn in (-1.0, 1.0):
        sites = []
        for j in range(p.na):
            o = np.zeros((2, 2, 2, 2), dtype=CT)
            o[0, :, 0, :] = I2
            o[0, :, 1, :] = 1j * np.sqrt(p.gam_1d[j] / 2) * np.exp(sgn * 1j * p.k_wg * p.rj[j]) * SM
            o[1, :, 1, :] = I2
            if j == 0:
                o = o[0:1]
                if sgn < 0:
                    o[0, :, 1, :] += p.f(t) * I2
            if j == p.na - 1:
                o = o[:, :, 1:2]
            sites.append(np.ascontiguousarray(o))
        out.append(sites)
    return out[0], out[1]


def _local_l(p, j, con, delt, t):
    g, ft = p.gam_1d[j], p.f(t)
    G = p.gam_eg + g
    k = np.kron
    X = SP + SM
    return con / p.na * k(I2, I2) + delt * (
        (1j * p.del_p - G / 2) * k(E_E, I2) - (1j * p.del_p + G / 2) * k(I2, E_E) + G * k(SM, SM)
        + 1j * ft * np.sqrt(g / 2) * np.exp(1j * p.k_in * p.rj[j]) * (k(SP, I2) - k(I2, SM))
        + 1j * ft * np.sqrt(g / 2) * np.exp(-1j * p.k_in * p.rj[j]) * (k(SM, I2) - k(I2, SP))
        + 1j * p.omega * (k(X, I2) - k(I2, X))
        + p.gam_phi * (k(E_E, E_E) - 0.5 * k(E_E, I2) - 0.5 * k(I2, E_E)))


def construct_L_spin_model(p, con, delt, t, w=6):
    """MPO of con*1 + delt*L for the vectorised density matrix (d=4), padded to width w >= 6."""
    na = p.na
    ph = np.exp(1j * p.k_wg * np.diff(p.rj))
    cp = np.sqrt(delt * p.gam_1d / 2)
    k = np.kron
    ii = k(I2, I2)
    W = max(6, int(w))
    last = W - 1
    out = []
    for j in range(na):
        o = np.zeros((W, 4, W, 4), dtype=CT)
        c = cp[j]
        if j < na - 1:
            q = ph[j]
            o[0, :, 0, :] = ii
            o[0, :, 1, :] = c * q * (k(I2, SM) - k(SP, I2))
            o[0, :, 2, :] = c * q * k(SM, I2)
            o[0, :, 3, :] = np.conj(c * q) * k(I2, SM)
            o[0, :, 4, :] = np.conj(c * q) * (k(SM, I2) - k(I2, SP))
            o[1, :, 1, :] = q * ii
            o[2, :, 2, :] = q * ii
            o[3, :, 3, :] = np.conj(q) * ii
            o[4, :, 4, :] = np.conj(q) * ii
        o[0, :, last, :] = _local_l(p, j, con, delt, t)
        o[1, :, last, :] = c * k(SM, I2)
        o[2, :, last, :] = -c * (k(SP, I2) - k(I2, SM))
        o[3, :, last, :] = -np.conj(c) * (k(I2, SP) - k(SM, I2))
        o[4, :, last, :] = np.conj(c) * k(I2, SM)
        o[last, :, last, :] = ii
        if j == 0:
            o = o[0:1]
        if j == na - 1:
            o = o[:, :, last:last + 1]
        out.append(np.ascontiguousarray(o))
    return out


# measurement functionals for a vectorised density matrix: Tr(X rho) = scal_prod_no_conj(X, rho)
TRACE_VEC = np.array([1, 0, 0, 1], dtype=CT)
SEE_VEC = np.array([0, 0, 0, 1], dtype=CT)
SP_VEC = np.array([0, 1, 0, 0], dtype=CT)
SM_VEC = np.array([0, 0, 1, 0], dtype=CT)


def functional_sites(na, site_vecs):
    """Product vectorised-operator MPS sites: ``site_vecs`` maps 0-based site -> length-4 vector."""
    return [np.asarray(site_vecs.get(j, TRACE_VEC), dtype=CT).reshape(1, 4, 1) for j in range(na)]


def product_mpo_sites(na, d, ops):
    """w=1 MPO sites with ``ops`` (0-based site -> d x d) and identity elsewhere."""
    return [np.asarray(ops.get(j, np.eye(d)), dtype=CT).reshape(1, d, 1, d) for j in range(na)]
