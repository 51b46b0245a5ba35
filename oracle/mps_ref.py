"""NumPy restatement of the MatrixProductStates.jl hot path (TEST INFRASTRUCTURE ONLY).

Conventions (shared with the reference, all column-major "Julia" semantics):

* site tensor      A[chiL, d, chiR]
* MPO site tensor  O[wL, d_out, wR, d_in]                    (src/constructors.jl:239-243)
* 3-index env      F[chi_A, w, chi_A0]; left envs are stored conjugated
                   (src/mps_base.jl:219-222)
* 2-index envs     FL[chi_A0, chi_A] (left), FR[chi_A, chi_A0] (right)

``jr(x, *shape)`` is Julia's ``reshape`` (column-major).  Every product below is
the same GEMM, with the same operands and transposes, as the cited Julia line;
QR goes through LAPACK ``zgeqrf`` + ``zungqr`` (numpy.linalg.qr), the routines
``qrq!`` calls (src/orthonormalisation.jl:180-184).

Julia's ``X[jj] = f(...)`` rebinding and ``f!(X[jj], ...)`` in-place writes are
both expressed here as list-slot assignment; the reference never reads an old
site array after it has been overwritten, so the two are equivalent.

PARITY UNPINNED: no reference output exists to pin this module (see package
docstring); it is validated against exact dense evolution instead.
"""
import numpy as np

CT = np.complex128


def jr(x, *shape):
    """Julia ``reshape(x, shape...)`` (column-major)."""
    return np.reshape(x, shape, order="F")


def ctr(x):
    """Julia ``x'`` (conjugate transpose) of a matrix."""
    return x.conj().T


# --------------------------------------------------------------------------
# src/mps_base.jl
# --------------------------------------------------------------------------

def prod_AOR(A, O, R):
    """src/mps_base.jl:7-19 -> AOR[chiL, wL, d_out, chiR0]."""
    a1, a2, a3 = A.shape
    _, r2, r3 = R.shape
    o1 = O.shape[0]
    AOR = jr(A, a1 * a2, a3) @ jr(R, a3, r2 * r3)
    AOR = np.transpose(jr(AOR, a1, a2, r2, r3), (2, 1, 0, 3))
    AOR = jr(O, o1 * a2, r2 * a2) @ jr(AOR, r2 * a2, a1 * r3)
    return np.transpose(jr(AOR, o1, a2, a1, r3), (2, 0, 1, 3))


def prod_AOL(A, O, L):
    """src/mps_base.jl:26-39 -> AOL[chiL0, d_out, chiR, wR] (uses L', conjugated storage)."""
    a1, d, a3 = A.shape
    _, l2, l3 = L.shape
    o3 = O.shape[2]
    AOL = ctr(jr(L, a1, l2 * l3)) @ jr(A, a1, d * a3)
    AOL = np.transpose(jr(AOL, l2, l3, d, a3), (1, 3, 0, 2))
    AOL = jr(AOL, l3 * a3, l2 * d)
    AOL = AOL @ jr(np.transpose(O, (0, 3, 1, 2)), l2 * d, d * o3)
    return np.transpose(jr(AOL, l3, a3, d, o3), (0, 2, 1, 3))


def prod_LR(L, R):
    """All ``prod_LR`` methods, dispatched on (ndims(L), ndims(R)) like Julia does.

    (3,4) src/mps_base.jl:45-51    L'-contraction with AOR
    (4,3) src/mps_base.jl:65-71    AOL times right env
    (2,3) src/mps_base.jl:85-90    2-index left env times site
    (3,2) src/mps_base.jl:122-127  site times 2-index right env
    """
    if L.ndim == 3 and R.ndim == 4:
        r1, r2, r3, r4 = R.shape
        l3 = L.shape[2]
        return jr(ctr(jr(L, r1 * r2, l3)) @ jr(R, r1 * r2, r3 * r4), l3, r3, r4)
    if L.ndim == 4 and R.ndim == 3:
        l1, l2, l3, l4 = L.shape
        r3 = R.shape[2]
        return jr(jr(L, l1 * l2, l3 * l4) @ jr(R, l3 * l4, r3), l1, l2, r3)
    if L.ndim == 2 and R.ndim == 3:
        r1, r2, r3 = R.shape
        return jr(L @ jr(R, r1, r2 * r3), L.shape[0], r2, r3)
    if L.ndim == 3 and R.ndim == 2:
        l1, l2, l3 = L.shape
        return jr(jr(L, l1 * l2, l3) @ R, l1, l2, R.shape[1])
    raise TypeError("no prod_LR method for ndims (%d, %d)" % (L.ndim, R.ndim))


def prod_LR_co(L, R):
    """src/mps_base.jl:92-97 (non-conjugate transpose of the 2-index env)."""
    r1, r2, r3 = R.shape
    return jr(L.T @ jr(R, r1, r2 * r3), L.shape[1], r2, r3)


def update_re(A0, AOR):
    """src/mps_base.jl:142-149 -> FR[chiL, wL, chiL0]."""
    r1, r2, r3, r4 = AOR.shape
    a1 = A0.shape[0]
    return jr(jr(AOR, r1 * r2, r3 * r4) @ ctr(jr(A0, a1, r3 * r4)), r1, r2, a1)


def update_re_full(A0, O, A, FR):
    """src/mps_base.jl:164-171 (update_re from A, O and A0)."""
    return update_re(A0, prod_AOR(A, O, FR))


def update_renv(A0, AR):
    """src/mps_base.jl:185-191 -> FR[chiL(A), chiL(A0)]."""
    a1, d, a2 = A0.shape
    return jr(AR, AR.shape[0], d * a2) @ ctr(jr(A0, a1, d * a2))


def update_renv_full(A0, A, FR):
    """src/mps_base.jl:204-210."""
    return update_renv(A0, prod_LR(A, FR))


def update_le(A0, AOL):
    """src/mps_base.jl:223-230 -> FL[chiR, wR, chiR0] (conjugated storage)."""
    l1, l2, l3, l4 = AOL.shape
    a3 = A0.shape[2]
    return jr(ctr(jr(AOL, l1 * l2, l3 * l4)) @ jr(A0, l1 * l2, a3), l3, l4, a3)


def update_le_full(A0, O, A, FL):
    """src/mps_base.jl:246-253."""
    return update_le(A0, prod_AOL(A, O, FL))


def update_lenv(A0, AL):
    """src/mps_base.jl:267-273 -> FL[chiR(A0), chiR(A)]."""
    a1, d, a3 = A0.shape
    return ctr(jr(A0, a1 * d, a3)) @ jr(AL, a1 * d, AL.shape[2])


def update_lenv_full(A0, A, L):
    """src/mps_base.jl:293-299."""
    return update_lenv(A0, prod_LR(L, A))


def update_lenv_nc(A0, AL):
    """src/mps_base.jl:319-325 (A0 not conjugated)."""
    a1, d, a3 = A0.shape
    return jr(A0, a1 * d, a3).T @ jr(AL, a1 * d, AL.shape[2])


def update_lenv_nc_full(A0, A, L):
    """src/mps_base.jl:330-336."""
    return update_lenv_nc(A0, prod_LR(L, A))


def local_exp(A0, A, O):
    """src/mps_base.jl:341-349: trace(O * (A_p * A0_p'))."""
    a1, d, a3 = A.shape
    Ap = jr(np.transpose(A, (1, 0, 2)), d, a1 * a3)
    A0p = jr(np.transpose(A0, (1, 0, 2)), d, a1 * a3)
    Ap = Ap @ ctr(A0p)
    return np.trace(O @ Ap)


# --------------------------------------------------------------------------
# src/orthonormalisation.jl
# --------------------------------------------------------------------------

def qrq(M):
    """src/orthonormalisation.jl:180-184: LAPACK geqrf + orgqr, Q only (thin)."""
    q = np.linalg.qr(np.asarray(M, dtype=CT), mode="reduced")[0]
    return q


def julia_qr(M):
    """Julia 0.6 ``qr(M)`` (thin Q, R) -- same Householder reflectors as geqrf."""
    q, r = np.linalg.qr(np.asarray(M, dtype=CT), mode="reduced")
    return q, r


def leftorth(A):
    """src/orthonormalisation.jl:150-157 -> (Q[Dl,d,k], C)."""
    Dl, d, Dr = A.shape
    Q, C = julia_qr(jr(A, d * Dl, Dr))
    return jr(Q, Dl, d, Q.shape[1]), C


def leftorth_(A):
    """src/orthonormalisation.jl:164-171 (``leftorth!``)."""
    Dl, d, Dr = A.shape
    Q = qrq(jr(A, d * Dl, Dr))
    return jr(Q, Dl, d, Q.shape[1])


def rightorth(A):
    """src/orthonormalisation.jl:204-211 -> (Q[k,d,Dr], C.')."""
    Dl, d, Dr = A.shape
    Q, C = julia_qr(jr(A, Dl, d * Dr).T)
    return jr(Q.T, Q.shape[1], d, Dr), C.T


def rightorth_(A):
    """src/orthonormalisation.jl:227-234 (``rightorth!``): QR of the non-conjugate transpose."""
    Dl, d, Dr = A.shape
    Q = qrq(jr(A, Dl, d * Dr).T)
    return jr(Q.T, Q.shape[1], d, Dr)


def leftorthogonalizeQR_(mps):
    """src/orthonormalisation.jl:43-56: left QR sweep carrying R, returns the norm^2."""
    n = len(mps)
    for i in range(n - 1):
        mps[i], r = leftorth(mps[i])
        mps[i + 1] = prod_LR(r, mps[i + 1])
    return float(np.sum(np.abs(mps[n - 1].ravel(order="F")) ** 2))


def leftorthonormalizationQR_(mps):
    """src/orthonormalisation.jl:29-36."""
    no = leftorthogonalizeQR_(mps)
    mps[-1] = mps[-1] / np.sqrt(no)
    return no


def rightorthogonalizeQR_(mps):
    """src/orthonormalisation.jl:77-90."""
    n = len(mps)
    for i in range(n - 1, 0, -1):
        mps[i], r = rightorth(mps[i])
        mps[i - 1] = prod_LR(mps[i - 1], r)
    return float(np.sum(np.abs(mps[0].ravel(order="F")) ** 2))


def normalize_lo_(mps):
    """src/orthonormalisation.jl:97-103: norm^2 from the last site, last site rescaled."""
    no = float(np.sum(np.abs(mps[-1].ravel(order="F")) ** 2))
    mps[-1] = mps[-1] / np.sqrt(no)
    return no


def norm_lo(mps):
    """src/orthonormalisation.jl:117-121."""
    return float(np.sum(np.abs(mps[-1].ravel(order="F")) ** 2))


# --------------------------------------------------------------------------
# src/constructors.jl
# --------------------------------------------------------------------------

def dims_rule(na, dmax, d):
    """Bond dims of src/constructors.jl:11-18: min(dmax, d^(k-1), d^(na+1-k))."""
    dims = [1] * (na + 1)
    for k in range(1, na):
        dims[k] = dmax
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
    return dims


def mpsproductstate(na, dmax, d, state):
    """src/constructors.jl:8-32 (``state`` a vector) and :37-61 (``state`` a callable of site 1..na)."""
    st = state if callable(state) else (lambda n: state)
    dims = [1] * (na + 1)
    for k in range(1, na):
        dims[k] = dmax
    r = np.ones((1, 1), dtype=CT)
    mps = [None] * na
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
        site = np.zeros((dims[n - 1], d, dims[n]), dtype=CT)
        site[0, :, 0] = np.asarray(st(n), dtype=CT)
        site = prod_LR(r, site)
        mps[n - 1], r = leftorth(site)
    site = np.zeros((dims[na - 1], d, dims[na]), dtype=CT)
    site[0, :, 0] = np.asarray(st(na), dtype=CT)
    mps[na - 1] = prod_LR(r, site)
    return mps, dims


def mpsgroundstate(na, dmax, d):
    """src/constructors.jl:69-75: product state with every site in basis state 1."""
    state = np.zeros(d, dtype=CT)
    state[0] = 1.0
    return mpsproductstate(na, dmax, d, state)


def crandn(rng, *shape):
    """``randn(Complex{Float64})`` of src/MatrixProductStates.jl:24-27 (SQRT_HALF*(re + i im)),
    drawn from an injected generator since Julia's stream cannot be reproduced here."""
    s = np.sqrt(0.5)
    re = rng.standard_normal(shape)
    im = rng.standard_normal(shape)
    return (s * re + 1j * s * im).astype(CT)


def mpsrandom(na, dmax, d, rng):
    """src/constructors.jl:113-129 with the normal draws taken from ``rng``.

    Each site is drawn column-major-contiguous (Julia fills arrays in memory order)."""
    dims = [1] * (na + 1)
    for k in range(1, na):
        dims[k] = dmax
    mps = [None] * na
    for n in range(1, na + 1):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
        shape = (dims[n - 1], d, dims[n])
        flat = crandn(rng, int(np.prod(shape)))
        mps[n - 1] = leftorth_(jr(flat, *shape))
    return mps, dims


def expandmps(mps, dmax):
    """src/constructors.jl:134-162: zero-pad to bond dim ``dmax`` and re-left-orthogonalise."""
    na = len(mps)
    d = mps[0].shape[1]
    dims = [dmax] * (na + 1)
    dims[0] = 1
    dims[na] = 1
    r = np.ones((1, 1), dtype=CT)
    out = [None] * na
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
        site = np.zeros((dims[n - 1], d, dims[n]), dtype=CT)
        a = mps[n - 1]
        site[: a.shape[0], :, : a.shape[2]] = a
        site = prod_LR(r, site)
        out[n - 1], r = leftorth(site)
    site = np.zeros((dims[na - 1], d, dims[na]), dtype=CT)
    a = mps[na - 1]
    site[: a.shape[0], :, : a.shape[2]] = a
    out[na - 1] = prod_LR(r, site)
    return out, dims


def makemps(mpsmat, na, d):
    """src/constructors.jl:200-222: ``mpsmat[l][m]`` is a callable of the site (1-based)."""
    b1 = len(mpsmat)
    b2 = len(mpsmat[0])
    mps = []
    for n in range(1, na + 1):
        site = np.zeros((b1, d, b2), dtype=CT)
        for m in range(b2):
            for l in range(b1):
                site[l, :, m] = np.asarray(mpsmat[l][m](n), dtype=CT)
        mps.append(site)
    mps[0] = mps[0][0:1, :, 0:b2].copy()
    mps[na - 1] = mps[na - 1][0:b1, :, b2 - 1:b2].copy()
    return mps


def makempo(mpomat, na, d):
    """src/constructors.jl:231-253: ``mpomat[l][m]`` is a callable of the site (1-based)."""
    b1 = len(mpomat)
    b2 = len(mpomat[0])
    mpo = []
    for n in range(1, na + 1):
        site = np.zeros((b1, d, b2, d), dtype=CT)
        for m in range(b2):
            for l in range(b1):
                site[l, :, m, :] = np.asarray(mpomat[l][m](n), dtype=CT) * np.ones((d, d))
        mpo.append(site)
    mpo[0] = mpo[0][0:1, :, 0:b2, :].copy()
    mpo[na - 1] = mpo[na - 1][0:b1, :, b2 - 1:b2, :].copy()
    return mpo


def mpo_to_mps_site(mpoin):
    """src/constructors.jl:310-315."""
    dl, d, dr, _ = mpoin.shape
    return jr(np.transpose(mpoin, (0, 1, 3, 2)), dl, d * d, dr)


def mpo_to_mps(mpoin):
    """src/constructors.jl:298-308."""
    return [mpo_to_mps_site(o) for o in mpoin]


def mpo_to_mps_dens_site(mpoin):
    """src/constructors.jl:336-341."""
    dl, d, dr, _ = mpoin.shape
    return jr(np.transpose(mpoin, (0, 3, 1, 2)), dl, d * d, dr)


def build_env(dims1, dims2, mpo_dims=None):
    """src/constructors.jl:347-375: N+1 env buffers, ones(1,1[,1]) at the two ends."""
    n1 = len(dims1)
    env = [None] * n1
    if mpo_dims is None:
        env[0] = np.ones((1, 1), dtype=CT)
        for n in range(1, n1 - 1):
            env[n] = np.zeros((dims1[n], dims2[n]), dtype=CT)
        env[n1 - 1] = np.ones((1, 1), dtype=CT)
    else:
        env[0] = np.ones((1, 1, 1), dtype=CT)
        for n in range(1, n1 - 1):
            env[n] = np.zeros((dims1[n], int(mpo_dims[n]), dims2[n]), dtype=CT)
        env[n1 - 1] = np.ones((1, 1, 1), dtype=CT)
    return env


# --------------------------------------------------------------------------
# src/MatrixProductStates.jl
# --------------------------------------------------------------------------

def apply_site_MPOtoMPO(mpo1, mpo2):
    """src/MatrixProductStates.jl:89-98 (operator product mpo2*mpo1 on one site)."""
    dwl1, d, dwr1, _ = mpo1.shape
    dwl2, _, dwr2, _ = mpo2.shape
    ai = jr(mpo2, dwl2 * d * dwr2, d) @ jr(np.transpose(mpo1, (1, 0, 2, 3)), d, dwl1 * dwr1 * d)
    ai = jr(ai, dwl2, d, dwr2, dwl1, dwr1, d)
    ai = np.transpose(ai, (3, 0, 1, 4, 2, 5))
    return jr(ai, dwl1 * dwl2, d, dwr1 * dwr2, d)


def applyMPOtoMPO(mpo1, mpo2):
    """src/MatrixProductStates.jl:67-76."""
    return [apply_site_MPOtoMPO(a, b) for a, b in zip(mpo1, mpo2)]


def conj_site_mpo(o):
    """src/MatrixProductStates.jl:409-413."""
    return np.transpose(o.conj(), (0, 3, 2, 1))


def conj_mpo(mpo):
    """src/MatrixProductStates.jl:395-406."""
    return [conj_site_mpo(o) for o in mpo]


def apply_site_MPOtoMPS(ms, mo):
    """src/MatrixProductStates.jl:126-133: ai[-1,-2,-3,-5,-4] = ms[-1,1,-5]*mo[-2,-3,-4,1]."""
    dl, _, dr = ms.shape
    dwl, d, dwr, _ = mo.shape
    # ai[a, w, s', b, w'] = sum_s ms[a, s, b] mo[w, s', w', s]
    ai = np.einsum("asb,wtvs->awtbv", ms, mo)
    return jr(ai, dl * dwl, d, dr * dwr)


def applyMPOtoMPS(mpsin, mpo):
    """src/MatrixProductStates.jl:115-124."""
    return [apply_site_MPOtoMPS(a, o) for a, o in zip(mpsin, mpo)]


def apply_site_operator_(mps_site, op):
    """src/MatrixProductStates.jl:135-143: returns op applied on the physical index."""
    m1, m2, m3 = mps_site.shape
    t = jr(np.transpose(mps_site, (1, 0, 2)), m2, m1 * m3)
    t = np.asarray(op, dtype=CT) @ t
    return np.transpose(jr(t, m2, m1, m3), (1, 0, 2)).copy()


def scal_op_prod(mps1, op, mps2):
    """src/MatrixProductStates.jl:327-340: <mps1|op|mps2>."""
    lenv = np.ones((1, 1, 1), dtype=CT)
    for i in range(len(mps1)):
        lenv = update_le_full(mps1[i], op[i], mps2[i], lenv)
    return complex(lenv.ravel()[0])


def scal_prod(mps1, mps2):
    """src/MatrixProductStates.jl:345-358: <mps1|mps2>."""
    lenv = np.ones((1, 1), dtype=CT)
    for n in range(len(mps1)):
        lenv = update_lenv_full(mps1[n], mps2[n], lenv)
    return complex(lenv.ravel()[0])


def scal_prod_no_conj(mps1, mps2):
    """src/MatrixProductStates.jl:366-379."""
    lenv = np.ones((1, 1), dtype=CT)
    for n in range(len(mps1)):
        lenv = update_lenv_nc_full(mps1[n], mps2[n], lenv)
    return complex(lenv.ravel()[0])


# --------------------------------------------------------------------------
# src/compression.jl (in-place apply-H family on the RK4 path)
# --------------------------------------------------------------------------

def _set_first(x, value):
    """``x[1] = value`` on a 1x1(x1) boundary env."""
    x = x.copy()
    x.reshape(-1, order="F")[0] = value
    return x


def compress_var_apply_H_(A0, envop, Ain, A, H, maxsweeps):
    """src/compression.jl:217-258: ``maxsweeps`` R->L/L->R sweep pairs of O*A into A0."""
    na = len(Ain)
    envop[0] = _set_first(envop[0], 1.0)
    for jj in range(na - 1):
        envop[jj + 1] = update_le_full(Ain[jj], H[jj], A[jj], envop[jj])
    envop[na] = _set_first(envop[na], 1.0)
    for _ in range(maxsweeps):
        for jj in range(na - 1, 0, -1):
            AOR = prod_AOR(A[jj], H[jj], envop[jj + 1])
            A0[jj] = prod_LR(envop[jj], AOR)
            A0[jj] = rightorth_(A0[jj])
            envop[jj] = update_re(A0[jj], AOR)
        for jj in range(na - 1):
            AOL = prod_AOL(A[jj], H[jj], envop[jj])
            A0[jj] = prod_LR(AOL, envop[jj + 1])
            A0[jj] = leftorth_(A0[jj])
            envop[jj + 1] = update_le(A0[jj], AOL)
        AOL = prod_AOL(A[na - 1], H[na - 1], envop[na - 1])
        A0[na - 1] = prod_LR(AOL, envop[na])


def compress_var_apply_H_left_(A0, envop, Ain, A, H):
    """src/compression.jl:321-347: left env init, then one R->L half sweep of O*A into A0."""
    na = len(Ain)
    envop[0] = _set_first(envop[0], 1.0)
    for jj in range(na - 1):
        envop[jj + 1] = update_le_full(Ain[jj], H[jj], A[jj], envop[jj])
    envop[na] = _set_first(envop[na], 1.0)
    for jj in range(na - 1, 0, -1):
        AOR = prod_AOR(A[jj], H[jj], envop[jj + 1])
        A0[jj] = prod_LR(envop[jj], AOR)
        A0[jj] = rightorth_(A0[jj])
        envop[jj] = update_re(A0[jj], AOR)
    AOR = prod_AOR(A[0], H[0], envop[1])
    A0[0] = prod_LR(envop[0], AOR)


def compress_sum_var_apply_H_(A0, envop, coef, A, H, maxsweeps):
    """src/compression.jl:805-887: sum_l coef[l] A[l] + coef[end] H*A[end] with full sweeps.

    A0 is both the guess (bra of the envs) and the output."""
    na = len(A0)
    numv = len(coef)
    env = []
    for ll in range(numv - 1):
        e = [None] * (na + 1)
        e[0] = np.ones((1, 1), dtype=CT)
        for jj in range(na - 1):
            e[jj + 1] = update_lenv_full(A0[jj], A[ll][jj], e[jj])
        e[na] = np.full((1, 1), coef[ll], dtype=CT)
        env.append(e)
    envop[0] = _set_first(envop[0], 1.0)
    for jj in range(na - 1):
        envop[jj + 1] = update_le_full(A0[jj], H[jj], A[numv - 1][jj], envop[jj])
    envop[na] = _set_first(envop[na], coef[numv - 1])
    AR = [None] * (numv - 1)
    for _ in range(maxsweeps):
        for jj in range(na - 1, 0, -1):
            AR[0] = prod_LR(A[0][jj], env[0][jj + 1])
            acc = prod_LR(env[0][jj], AR[0])
            for ll in range(1, numv - 1):
                AR[ll] = prod_LR(A[ll][jj], env[ll][jj + 1])
                acc = acc + prod_LR(env[ll][jj], AR[ll])
            AOR = prod_AOR(A[numv - 1][jj], H[jj], envop[jj + 1])
            acc = acc + prod_LR(envop[jj], AOR)
            A0[jj] = rightorth_(acc)
            for ll in range(numv - 1):
                env[ll][jj] = update_renv(A0[jj], AR[ll])
            envop[jj] = update_re(A0[jj], AOR)
        for jj in range(na - 1):
            AR[0] = prod_LR(env[0][jj], A[0][jj])
            acc = prod_LR(AR[0], env[0][jj + 1])
            for ll in range(1, numv - 1):
                AR[ll] = prod_LR(env[ll][jj], A[ll][jj])
                acc = acc + prod_LR(AR[ll], env[ll][jj + 1])
            AOL = prod_AOL(A[numv - 1][jj], H[jj], envop[jj])
            acc = acc + prod_LR(AOL, envop[jj + 1])
            A0[jj] = leftorth_(acc)
            for ll in range(numv - 1):
                env[ll][jj + 1] = update_lenv(A0[jj], AR[ll])
            envop[jj + 1] = update_le(A0[jj], AOL)
    AR[0] = prod_LR(env[0][na - 1], A[0][na - 1])
    acc = prod_LR(AR[0], env[0][na])
    for ll in range(1, numv - 1):
        AR[ll] = prod_LR(env[ll][na - 1], A[ll][na - 1])
        acc = acc + prod_LR(AR[ll], env[ll][na])
    AOL = prod_AOL(A[numv - 1][na - 1], H[na - 1], envop[na - 1])
    A0[na - 1] = acc + prod_LR(AOL, envop[na])


def compress_sum_var(Ain, coef, A, maxsweeps):
    """src/compression.jl:496-565: returns the compression of sum_l coef[l] A[l], guess Ain."""
    na = len(Ain)
    numv = len(coef)
    FL, FR = [], []
    for ll in range(numv):
        fl = [None] * na
        fl[0] = np.ones((1, 1), dtype=CT)
        for jj in range(na - 1):
            fl[jj + 1] = update_lenv_full(Ain[jj], A[ll][jj], fl[jj])
        fr = [None] * na
        fr[na - 1] = np.full((1, 1), coef[ll], dtype=CT)
        FL.append(fl)
        FR.append(fr)
    A0 = [None] * na
    AR = [None] * numv
    for _ in range(maxsweeps):
        for jj in range(na - 1, 0, -1):
            AR[0] = prod_LR(A[0][jj], FR[0][jj])
            acc = prod_LR(FL[0][jj], AR[0])
            for ll in range(1, numv):
                AR[ll] = prod_LR(A[ll][jj], FR[ll][jj])
                acc = acc + prod_LR(FL[ll][jj], AR[ll])
            A0[jj] = rightorth_(acc)
            for ll in range(numv):
                FR[ll][jj - 1] = update_renv(A0[jj], AR[ll])
        for jj in range(na - 1):
            AR[0] = prod_LR(FL[0][jj], A[0][jj])
            acc = prod_LR(AR[0], FR[0][jj])
            for ll in range(1, numv):
                AR[ll] = prod_LR(FL[ll][jj], A[ll][jj])
                acc = acc + prod_LR(AR[ll], FR[ll][jj])
            A0[jj] = leftorth_(acc)
            for ll in range(numv):
                FL[ll][jj + 1] = update_lenv(A0[jj], AR[ll])
    AR[0] = prod_LR(FL[0][na - 1], A[0][na - 1])
    acc = prod_LR(AR[0], FR[0][na - 1])
    for ll in range(1, numv):
        AR[ll] = prod_LR(FL[ll][na - 1], A[ll][na - 1])
        acc = acc + prod_LR(AR[ll], FR[ll][na - 1])
    A0[na - 1] = acc
    return A0


def Arnoldi_expm_(A, rhov, numv, env, envop):
    """src/timeevolution.jl:88-119 (rhov[0] <- normalised Krylov approximation of exp(A) rhov[0]).

    Returns coef = expm(N \\ H)[:, 0]; `env` is unused, as in the reference."""
    import scipy.linalg
    Nm = np.eye(numv, dtype=CT)
    Hm = np.zeros((numv, numv), dtype=CT)
    Hm[0, 0] = scal_op_prod(rhov[0], A, rhov[0])
    for jj in range(1, numv):
        coef = [-Hm[ll, jj - 1] for ll in range(jj)] + [1.0]
        compress_sum_var_apply_H_(rhov[jj], envop, coef, list(rhov[:jj]) + [rhov[jj - 1]], A, 1)
        normalize_lo_(rhov[jj])
        Hm[jj, jj] = scal_op_prod(rhov[jj], A, rhov[jj])
        for ll in range(jj):
            Hm[jj, ll] = scal_op_prod(rhov[jj], A, rhov[ll])
            Hm[ll, jj] = scal_op_prod(rhov[ll], A, rhov[jj])
            Nm[jj, ll] = scal_prod(rhov[jj], rhov[ll])
            Nm[ll, jj] = np.conj(Nm[jj, ll])
    coef = scipy.linalg.expm(np.linalg.solve(Nm, Hm))[:, 0]
    rhov[0] = compress_sum_var(rhov[0], coef, rhov, 1)
    normalize_lo_(rhov[0])
    return coef


def compress_sum_var_apply_H_left_(A0, env, envop, Ain, coef, A, H):
    """src/compression.jl:889-944: stage with an R->L half sweep (coefficients in the right boundary)."""
    na = len(Ain)
    numv = len(coef)
    for ll in range(numv - 1):
        env[ll][0] = _set_first(env[ll][0], 1.0)
        for jj in range(na - 1):
            env[ll][jj + 1] = update_lenv_full(Ain[jj], A[ll][jj], env[ll][jj])
        env[ll][na] = _set_first(env[ll][na], coef[ll])
    envop[0] = _set_first(envop[0], 1.0)
    for jj in range(na - 1):
        envop[jj + 1] = update_le_full(Ain[jj], H[jj], A[numv - 1][jj], envop[jj])
    envop[na] = _set_first(envop[na], coef[numv - 1])
    AR = [None] * (numv - 1)
    for jj in range(na - 1, 0, -1):
        AR[0] = prod_LR(A[0][jj], env[0][jj + 1])
        acc = prod_LR(env[0][jj], AR[0])
        for ll in range(1, numv - 1):
            AR[ll] = prod_LR(A[ll][jj], env[ll][jj + 1])
            acc = acc + prod_LR(env[ll][jj], AR[ll])
        AOR = prod_AOR(A[numv - 1][jj], H[jj], envop[jj + 1])
        acc = acc + prod_LR(envop[jj], AOR)
        A0[jj] = rightorth_(acc)
        for ll in range(numv - 1):
            env[ll][jj] = update_renv(A0[jj], AR[ll])
        envop[jj] = update_re(A0[jj], AOR)
    AR[0] = prod_LR(A[0][0], env[0][1])
    acc = prod_LR(env[0][0], AR[0])
    for ll in range(1, numv - 1):
        AR[ll] = prod_LR(A[ll][0], env[ll][1])
        acc = acc + prod_LR(env[ll][0], AR[ll])
    AOR = prod_AOR(A[numv - 1][0], H[0], envop[1])
    A0[0] = acc + prod_LR(envop[0], AOR)


def compress_sum_var_apply_H_right_(A0, env, envop, Ain, coef, A, H):
    """src/compression.jl:1007-1063: stage with an L->R half sweep (coefficients in the left boundary)."""
    na = len(Ain)
    numv = len(coef)
    for ll in range(numv - 1):
        env[ll][na] = _set_first(env[ll][na], 1.0)
        for jj in range(na - 1, 0, -1):
            env[ll][jj] = update_renv_full(Ain[jj], A[ll][jj], env[ll][jj + 1])
        env[ll][0] = _set_first(env[ll][0], coef[ll])
    envop[na] = _set_first(envop[na], 1.0)
    for jj in range(na - 1, 0, -1):
        envop[jj] = update_re_full(Ain[jj], H[jj], A[numv - 1][jj], envop[jj + 1])
    envop[0] = _set_first(envop[0], coef[numv - 1])
    AL = [None] * (numv - 1)
    for jj in range(na - 1):
        AL[0] = prod_LR(env[0][jj], A[0][jj])
        acc = prod_LR(AL[0], env[0][jj + 1])
        for ll in range(1, numv - 1):
            AL[ll] = prod_LR(env[ll][jj], A[ll][jj])
            acc = acc + prod_LR(AL[ll], env[ll][jj + 1])
        AOL = prod_AOL(A[numv - 1][jj], H[jj], envop[jj])
        acc = acc + prod_LR(AOL, envop[jj + 1])
        A0[jj] = leftorth_(acc)
        for ll in range(numv - 1):
            env[ll][jj + 1] = update_lenv(A0[jj], AL[ll])
        envop[jj + 1] = update_le(A0[jj], AOL)
    AL[0] = prod_LR(env[0][na - 1], A[0][na - 1])
    acc = prod_LR(AL[0], env[0][na])
    for ll in range(1, numv - 1):
        AL[ll] = prod_LR(env[ll][na - 1], A[ll][na - 1])
        acc = acc + prod_LR(AL[ll], env[ll][na])
    AOL = prod_AOL(A[numv - 1][na - 1], H[na - 1], envop[na - 1])
    A0[na - 1] = acc + prod_LR(AOL, envop[na])


# --------------------------------------------------------------------------
# src/timeevolution.jl
# --------------------------------------------------------------------------

def RK4stp_apply_H_half_(dt, H, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop):
    """src/timeevolution.jl:178-196.

    The 10-argument (in-place) form is ``psi0 is psi``; the 11-argument form passes a
    separate output list.  Stage coefficients [1,dt/2], [1,dt], [-1/3,1/3,2/3,1/3]."""
    compress_var_apply_H_left_(psi1, envop, psi, psi, H[0])
    compress_sum_var_apply_H_right_(psi2, [env1], envop, psi1, [1.0, dt / 2], [psi, psi1], H[1])
    compress_sum_var_apply_H_left_(psi3, [env1], envop, psi2, [1.0, dt], [psi, psi2], H[1])
    compress_sum_var_apply_H_right_(psi0, [env1, env2, env3], envop, psi3,
                                    [-1.0 / 3, 1.0 / 3, 2.0 / 3, 1.0 / 3],
                                    [list(psi), psi1, psi2, psi3], H[2])


def compressionSVD_(mps, dmax, tol=1e-15):
    """src/compression.jl:1280-1312: right-to-left SVD truncation of a left-canonical MPS
    (mps replaced site by site, bonds shrink); returns (err_glob, err_trim, ent_ent)."""
    n = len(mps)
    err_trim = np.zeros(n)
    ent_ent = np.zeros(n)
    dnew = 1
    r = np.ones((1, 1), dtype=CT)
    for i in range(n - 1, -1, -1):
        dl, d, dr = mps[i].shape
        mps_site = jr(mps[i], dl * d, dr) @ r
        u, s, vh = np.linalg.svd(jr(mps_site, dl, dnew * d), full_matrices=False)
        s = s[s > 0]
        stot = np.sum(s ** 2)
        b = dnew
        dnew = min(int(np.sum(np.cumsum(s ** 2 / stot) < (1 - tol))) + 1, dmax)
        err_trim[i] = np.sum(s[dnew:] ** 2) / stot
        ent_ent[i] = -2 * np.sum(s ** 2 * np.log(s))
        v = vh.conj().T
        mps[i] = jr(v[:, :dnew].conj().T, dnew, d, b)
        r = u[:, :dnew] @ np.diag(s[:dnew])
    err_glob = 1 - abs(r[0, 0]) ** 2
    return err_glob, err_trim, ent_ent


def _trunc_rule(s, tol, dlim):
    s = s[s > 0]
    stot = np.sum(s ** 2)
    return min(int(np.sum(np.cumsum(s ** 2 / stot) < 1 - tol)) + 1, dlim, len(s))


def compress_var_apply_H_two_site(Ain, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:355-411 with its `svdecon` (undefined in the reference) as the thin
    SVD, and the pair tensor contracted with the conjugated left environment like every
    single-site contraction: av = sum conj(L) A1 O1 A2 O2 R.  dims is updated in place."""
    na = len(Ain)
    FL, FR = [None] * na, [None] * na
    FL[0] = np.ones((1, 1, 1), dtype=CT)
    for jj in range(na - 2):
        FL[jj + 1] = update_le_full(Ain[jj], H[jj], A[jj], FL[jj])
    FR[na - 1] = np.ones((1, 1, 1), dtype=CT)
    A0 = [None] * na
    d = A[0].shape[1]

    def pair(j):
        X = prod_AOR(A[j + 1], H[j + 1], FR[j + 1])                       # [c, v, s2, b0]
        R2 = X.reshape(X.shape[0], X.shape[1], -1, order="F")              # [c, v, (s2 b0)]
        Y = prod_AOR(A[j], H[j], R2)                                       # [a, w, s1, (s2 b0)]
        av = np.einsum("awx,awsy->xsy", FL[j].conj(), Y)
        return av.reshape(av.shape[0] * d, -1, order="F")

    for _ in range(maxsweeps):
        for j in range(na - 2, -1, -1):
            u, s, vh = np.linalg.svd(pair(j), full_matrices=False)
            dn = _trunc_rule(s, svd_tol, dlim)
            dims[j + 1] = dn
            A0[j + 1] = jr(vh[:dn, :], dn, d, dims[j + 2])
            FR[j] = update_re_full(A0[j + 1], H[j + 1], A[j + 1], FR[j + 1])
        for j in range(na - 1):
            u, s, vh = np.linalg.svd(pair(j), full_matrices=False)
            dn = _trunc_rule(s, svd_tol, dlim)
            dims[j + 1] = dn
            A0[j] = jr(u[:, :dn], dims[j], d, dn)
            FL[j + 1] = update_le_full(A0[j], H[j], A[j], FL[j])
        A0[na - 1] = jr(np.diag(s[:dn]) @ vh[:dn, :], dn, d, dims[na])
    return A0


def compress_sum_var_apply_H_two_site(Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim, mode=0):
    """src/compression.jl:1072-1157 (mode 0), its _left form :1159-1215 (mode 1: one R->L
    sweep, first site U diag(S)) and _right form :1218-1276 (mode 2: one L->R sweep from right
    environments of a right-canonical Ain, coefficients on the left boundary); with H None,
    compress_sum_var_two_site :574-648 (every term plain).  The pair tensor is
    sum_l FL_l A_l1 A_l2 FR_l + sum conj(L) A1 O1 A2 O2 R with the 2-index left environment
    contracted on its A index (the single-site convention; the reference's
    A_prod_LR_two_site, src/MatrixProductStates.jl:288-292, contracts it transposed) and
    `svdecon` as the thin SVD.  dims is updated in place."""
    na = len(Ain)
    numv = len(coef)
    np_ = numv - 1 if H is not None else numv
    AH = A[numv - 1]
    d = AH[0].shape[1]
    one2 = np.ones((1, 1), dtype=CT)
    one3 = np.ones((1, 1, 1), dtype=CT)
    FL2 = [[None] * (na + 1) for _ in range(np_)]
    FR2 = [[None] * (na + 1) for _ in range(np_)]
    FL, FR = [None] * (na + 1), [None] * (na + 1)
    for l in range(np_):
        FL2[l][0] = coef[l] * one2 if mode == 2 else one2
        FR2[l][na] = one2 if mode == 2 else coef[l] * one2
    if H is not None:
        # the 3-index left environment is stored conjugated: conj(coef) there applies coef
        FL[0] = np.conj(coef[-1]) * one3 if mode == 2 else one3
        FR[na] = one3 if mode == 2 else coef[-1] * one3
    A0 = copy_mps(Ain)

    def left_update(k):                       # FL[k+1] from A0[k]
        for l in range(np_):
            FL2[l][k + 1] = update_lenv_full(A0[k], A[l][k], FL2[l][k])
        if H is not None:
            FL[k + 1] = update_le_full(A0[k], H[k], AH[k], FL[k])

    def right_update(k):                      # FR[k] from A0[k]
        for l in range(np_):
            FR2[l][k] = update_renv_full(A0[k], A[l][k], FR2[l][k + 1])
        if H is not None:
            FR[k] = update_re_full(A0[k], H[k], AH[k], FR[k + 1])

    if mode == 2:
        for k in range(na - 1, 1, -1):
            right_update(k)
    else:
        for k in range(na - 2):
            left_update(k)

    def pair(j):
        av = 0
        for l in range(np_):
            t = np.einsum("xa,asc,ctb,by->xsty", FL2[l][j], A[l][j], A[l][j + 1], FR2[l][j + 2])
            av = av + t.reshape(t.shape[0], d, -1, order="F")
        if H is not None:
            X = prod_AOR(AH[j + 1], H[j + 1], FR[j + 2])
            R2 = X.reshape(X.shape[0], X.shape[1], -1, order="F")
            Y = prod_AOR(AH[j], H[j], R2)
            av = av + np.einsum("awx,awsy->xsy", FL[j].conj(), Y)
        return av.reshape(av.shape[0] * d, -1, order="F")

    def sweep_left():
        out = None
        for j in range(na - 2, -1, -1):
            u, s, vh = np.linalg.svd(pair(j), full_matrices=False)
            dn = _trunc_rule(s, svd_tol, dlim)
            dims[j + 1] = dn
            A0[j + 1] = jr(vh[:dn, :], dn, d, dims[j + 2])
            right_update(j + 1)
            out = (u, s, dn)
        return out

    def sweep_right():
        out = None
        for j in range(na - 1):
            u, s, vh = np.linalg.svd(pair(j), full_matrices=False)
            dn = _trunc_rule(s, svd_tol, dlim)
            dims[j + 1] = dn
            A0[j] = jr(u[:, :dn], dims[j], d, dn)
            left_update(j)
            out = (s, vh, dn)
        return out

    if mode == 0:
        for _ in range(maxsweeps):
            sweep_left()
            s, vh, dn = sweep_right()
            A0[na - 1] = jr(np.diag(s[:dn]) @ vh[:dn, :], dn, d, dims[na])
    elif mode == 1:
        u, s, dn = sweep_left()
        A0[0] = jr(u[:, :dn] @ np.diag(s[:dn]), dims[0], d, dn)
    else:
        s, vh, dn = sweep_right()
        A0[na - 1] = jr(np.diag(s[:dn]) @ vh[:dn, :], dn, d, dims[na])
    return A0


def compress_var_apply_H_two_site_left(Ain, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:413-448: the single-term one R->L two-site sweep."""
    return compress_sum_var_apply_H_two_site(Ain, [1.0], [A], H, maxsweeps, svd_tol, dims, dlim, 1)


def compress_var_apply_H_two_site_right(Ain, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:450-486: the single-term one L->R two-site sweep."""
    return compress_sum_var_apply_H_two_site(Ain, [1.0], [A], H, maxsweeps, svd_tol, dims, dlim, 2)


def RK4stp_apply_H_half_full_two_site(dt, H, psi, svd_tol, dims, dlim):
    """src/timeevolution.jl:208-215: the RK4 step with every stage a two-site half sweep, the
    bond dims adapting (dims updated in place); returns the new psi."""
    psi1 = compress_var_apply_H_two_site_left(psi, psi, H[0], 1, svd_tol, dims, dlim)
    psi2 = compress_sum_var_apply_H_two_site(psi1, [1, dt / 2], [psi, psi1], H[1], 1, svd_tol, dims, dlim, 2)
    psi3 = compress_sum_var_apply_H_two_site(psi2, [1, dt], [psi, psi2], H[1], 1, svd_tol, dims, dlim, 1)
    return compress_sum_var_apply_H_two_site(psi3, [-1 / 3, 1 / 3, 2 / 3, 1 / 3], [psi, psi1, psi2, psi3], H[2], 1,
                                             svd_tol, dims, dlim, 2)


def copy_mps(mps):
    return [np.array(a, dtype=CT, copy=True) for a in mps]
