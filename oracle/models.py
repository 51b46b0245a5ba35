"""Spin-model MPO builders restated from the reference examples (TEST INFRASTRUCTURE ONLY).

* ``sm_hamiltonian``          examples/spin_model_quantum_trajectory_rk4.jl:235-271 (w=4, d=2)
* ``update_h``                examples/spin_model_quantum_trajectory_rk4.jl:274-284
* ``local_h``                 examples/spin_model_quantum_trajectory_rk4.jl:287-293
* ``jump_mpos``               examples/spin_model_quantum_trajectory_rk4.jl:51-55
* ``construct_L_spin_model``  examples/spin_model_density_matrix.jl:245-290 (w=6, d=4)
* ``local_l``                 examples/spin_model_density_matrix.jl:306-317

Two terms that the benchmark workloads name are added to the local terms and are
zero by default, so the builders reduce exactly to the examples:

* ``omega``   a Hermitian drive H_d = -omega (sigma+ + sigma-) on every site
* ``gam_phi`` pure dephasing, Lindblad operator sqrt(gam_phi) sigma_ee (density matrix only)

Basis per atom is [g, e] (index 1 = g); hge = |g><e| = sigma-, heg = sigma+.
A vectorised density matrix uses the site basis [gg, ge, eg, ee] and
``kron(X, Y) vec(rho) = vec(X rho Y^T)`` (examples/spin_model_density_matrix.jl:39-45).
"""
import numpy as np

from . import mps_ref as R

CT = np.complex128
hgg = np.array([[1, 0], [0, 0]], dtype=CT)
hee = np.array([[0, 0], [0, 1]], dtype=CT)
hge = np.array([[0, 1], [0, 0]], dtype=CT)
heg = hge.conj().T.copy()
id2 = np.eye(2, dtype=CT)


class SpinChain:
    """Parameters of the waveguide spin model (the ``const`` globals of the examples)."""

    def __init__(self, na, gam_1d=1.0, gam_eg=0.0, del_p=0.0, k_wg=0.5 * np.pi,
                 rj=None, k_in=0.5 * np.pi, f=None, omega=0.0, gam_phi=0.0):
        self.na = na
        self.gam_1d = np.full(na, float(gam_1d)) if np.isscalar(gam_1d) else np.asarray(gam_1d, float)
        self.gam_eg = float(gam_eg)
        self.del_p = float(del_p)
        self.k_wg = float(k_wg)
        self.rj = np.arange(1.0, na + 1.0) if rj is None else np.asarray(rj, float)
        self.k_in = float(k_in)
        self.f = f if f is not None else (lambda t: 0.0)
        self.omega = float(omega)
        self.gam_phi = float(gam_phi)


def local_h(p, jj, con, delt, time):
    """Local term of the trajectory generator (jj is 1-based), plus the ``omega`` drive."""
    g = p.gam_1d[jj - 1]
    ft = p.f(time)
    return (con * id2 / p.na
            + delt * ((1j * p.del_p - (p.gam_eg + g) / 2) * hee
                      + 1j * np.sqrt(g / 2) * ft * np.exp(1j * p.k_in * p.rj[jj - 1]) * heg
                      - (1.0 / (2 * p.na)) * abs(ft) ** 2 * id2
                      + 1j * p.omega * (heg + hge)))


def sm_hamiltonian(p, con, delt, time):
    """w=4 MPO of 1*con + delt*(-i H_eff) for the waveguide spin chain."""
    na = p.na
    drj = np.diff(p.rj)
    ph = np.exp(1j * p.k_wg * drj)
    cp = np.sqrt(delt * p.gam_1d / 2)
    H = [None] * na
    H[0] = np.zeros((1, 2, 4, 2), dtype=CT)
    H[0][0, :, 0, :] = id2
    H[0][0, :, 1, :] = -cp[0] * ph[0] * heg
    H[0][0, :, 2, :] = -cp[0] * ph[0] * hge
    H[0][0, :, 3, :] = local_h(p, 1, con, delt, time)
    H[na - 1] = np.zeros((4, 2, 1, 2), dtype=CT)
    H[na - 1][0, :, 0, :] = local_h(p, na, con, delt, time)
    H[na - 1][1, :, 0, :] = cp[na - 1] * hge
    H[na - 1][2, :, 0, :] = cp[na - 1] * heg
    H[na - 1][3, :, 0, :] = id2
    for jj in range(2, na):
        h = np.zeros((4, 2, 4, 2), dtype=CT)
        h[0, :, 0, :] = id2
        h[0, :, 1, :] = -cp[jj - 1] * ph[jj - 1] * heg
        h[0, :, 2, :] = -cp[jj - 1] * ph[jj - 1] * hge
        h[0, :, 3, :] = local_h(p, jj, con, delt, time)
        h[1, :, 3, :] = cp[jj - 1] * hge
        h[2, :, 3, :] = cp[jj - 1] * heg
        h[1, :, 1, :] = ph[jj - 1] * id2
        h[2, :, 2, :] = ph[jj - 1] * id2
        h[3, :, 3, :] = id2
        H[jj - 1] = h
    return H


def update_h(H, p, con, delt, time):
    """In-place local-term refresh for a time-dependent drive."""
    na = p.na
    H[0][0, :, 3, :] = local_h(p, 1, con, delt, time)
    H[na - 1][0, :, 0, :] = local_h(p, na, con, delt, time)
    for jj in range(2, na):
        H[jj - 1][0, :, 3, :] = local_h(p, jj, con, delt, time)


def jump_mpos(p, time=0.0):
    """(jumpright, jumpleft) w=2 MPOs of the waveguide output operators."""
    na, d = p.na, 2
    g, k, r = p.gam_1d, p.k_wg, p.rj
    jl = R.makempo([[lambda jj: id2, lambda jj: 1j * np.sqrt(g[jj - 1] / 2) * np.exp(1j * k * r[jj - 1]) * hge],
                    [lambda jj: 0, lambda jj: id2]], na, d)
    jr_ = R.makempo([[lambda jj: id2, lambda jj: 1j * np.sqrt(g[jj - 1] / 2) * np.exp(-1j * k * r[jj - 1]) * hge],
                     [lambda jj: 0, lambda jj: id2]], na, d)
    jr_[0][0, :, 1, :] = p.f(time) * id2 + 1j * np.sqrt(g[0] / 2) * np.exp(-1j * k * r[0]) * hge
    return jr_, jl


def local_l(p, jj, con, delt, time):
    """Local Lindbladian term (jj 1-based), plus the ``omega`` drive and ``gam_phi`` dephasing."""
    g = p.gam_1d[jj - 1]
    ft = p.f(time)
    G = p.gam_eg + g
    X = heg + hge
    return (con / p.na * np.kron(id2, id2)
            + delt * ((1j * p.del_p - G / 2) * np.kron(hee, id2)
                      - (1j * p.del_p + G / 2) * np.kron(id2, hee)
                      + G * np.kron(hge, hge)
                      + 1j * ft * np.sqrt(g / 2) * np.exp(1j * p.k_in * p.rj[jj - 1])
                      * (np.kron(hge.conj().T, id2) - np.kron(id2, hge))
                      + 1j * ft * np.sqrt(g / 2) * np.exp(-1j * p.k_in * p.rj[jj - 1])
                      * (np.kron(hge, id2) - np.kron(id2, hge.conj().T))
                      + 1j * p.omega * (np.kron(X, id2) - np.kron(id2, X))
                      + p.gam_phi * (np.kron(hee, hee) - 0.5 * np.kron(hee, id2) - 0.5 * np.kron(id2, hee))))


def construct_L_spin_model(p, con, delt, time, w=6):
    """w=6 Lindbladian MPO of con*1 + delt*L; ``w>6`` appends zero channels before the last one."""
    na = p.na
    drj = np.diff(p.rj)
    ph = np.exp(1j * p.k_wg * drj)
    cp = np.sqrt(delt * p.gam_1d / 2)
    ii = np.kron(id2, id2)
    hp = hge.conj().T
    L = [None] * na
    L[0] = np.zeros((1, 4, 6, 4), dtype=CT)
    L[0][0, :, 0, :] = ii
    L[0][0, :, 1, :] = cp[0] * ph[0] * (np.kron(id2, hge) - np.kron(hp, id2))
    L[0][0, :, 2, :] = cp[0] * ph[0] * np.kron(hge, id2)
    L[0][0, :, 3, :] = np.conj(cp[0]) * np.conj(ph[0]) * np.kron(id2, hge)
    L[0][0, :, 4, :] = np.conj(cp[0]) * np.conj(ph[0]) * (np.kron(hge, id2) - np.kron(id2, hp))
    L[0][0, :, 5, :] = local_l(p, 1, con, delt, time)
    L[na - 1] = np.zeros((6, 4, 1, 4), dtype=CT)
    L[na - 1][0, :, 0, :] = local_l(p, na, con, delt, time)
    L[na - 1][1, :, 0, :] = cp[na - 1] * np.kron(hge, id2)
    L[na - 1][2, :, 0, :] = -cp[na - 1] * (np.kron(hp, id2) - np.kron(id2, hge))
    L[na - 1][3, :, 0, :] = -np.conj(cp[na - 1]) * (np.kron(id2, hp) - np.kron(hge, id2))
    L[na - 1][4, :, 0, :] = np.conj(cp[na - 1]) * np.kron(id2, hge)
    L[na - 1][5, :, 0, :] = ii
    for jj in range(2, na):
        m = np.zeros((6, 4, 6, 4), dtype=CT)
        c, q = cp[jj - 1], ph[jj - 1]
        m[0, :, 0, :] = ii
        m[0, :, 1, :] = c * q * (np.kron(id2, hge) - np.kron(hp, id2))
        m[0, :, 2, :] = c * q * np.kron(hge, id2)
        m[0, :, 3, :] = np.conj(c) * np.conj(q) * np.kron(id2, hge)
        m[0, :, 4, :] = np.conj(c) * np.conj(q) * (np.kron(hge, id2) - np.kron(id2, hp))
        m[0, :, 5, :] = local_l(p, jj, con, delt, time)
        m[1, :, 5, :] = c * np.kron(hge, id2)
        m[2, :, 5, :] = -c * (np.kron(hp, id2) - np.kron(id2, hge))
        m[3, :, 5, :] = -np.conj(c) * (np.kron(id2, hp) - np.kron(hge, id2))
        m[4, :, 5, :] = np.conj(c) * np.kron(id2, hge)
        m[5, :, 5, :] = ii
        m[1, :, 1, :] = q * ii
        m[2, :, 2, :] = q * ii
        m[3, :, 3, :] = np.conj(q) * ii
        m[4, :, 4, :] = np.conj(q) * ii
        L[jj - 1] = m
    if w > 6:
        L = pad_mpo(L, w)
    return L


def pad_mpo(mpo, w):
    """Append ``w - w0`` zero channels to an upper-triangular MPO, keeping the last channel last."""
    na = len(mpo)
    out = []
    for n, o in enumerate(mpo):
        wl, d, wr, _ = o.shape
        nl = 1 if n == 0 else w
        nr = 1 if n == na - 1 else w
        x = np.zeros((nl, d, nr, d), dtype=CT)
        li = [0] if n == 0 else list(range(wl - 1)) + [w - 1]
        ri = [0] if n == na - 1 else list(range(wr - 1)) + [w - 1]
        for a, aa in enumerate(li):
            for b, bb in enumerate(ri):
                x[aa, :, bb, :] = o[a, :, b, :]
        out.append(x)
    return out


# ---- measurement MPS/MPOs ---------------------------------------------------

def identity_lmps(na):
    """IDlmps of examples/spin_model_density_matrix.jl:48: vec(1) on every site."""
    return R.makemps([[lambda jj: np.array([1, 0, 0, 1])]], na, 4)


def rho_site_functional_lmps(na, site_vecs):
    """Product vectorised-operator MPS: ``site_vecs`` maps 1-based site -> length-4 vector,
    identity (vec(1)) elsewhere; ``scal_prod_no_conj`` with it gives Tr(X rho)."""
    out = identity_lmps(na)
    for j, v in site_vecs.items():
        out[j - 1] = np.asarray(v, dtype=CT).reshape(1, 4, 1)
    return out


SEE_VEC = np.array([0, 0, 0, 1])   # Tr(sigma_ee rho_site) = rho_ee
SP_VEC = np.array([0, 1, 0, 0])    # Tr(sigma+ rho_site)  = rho_ge
SM_VEC = np.array([0, 0, 1, 0])    # Tr(sigma- rho_site)  = rho_eg


def product_mpo(na, d, ops):
    """w=1 MPO with ``ops`` (1-based site -> d x d) and identity elsewhere."""
    out = []
    for j in range(1, na + 1):
        o = np.asarray(ops.get(j, np.eye(d)), dtype=CT)
        out.append(o.reshape(1, d, 1, d))
    return out
