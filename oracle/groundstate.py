"""Oracle (test infrastructure only): ground_state_search! / steady_state_search! and their
effective-operator contractions, restated in NumPy.

  * A_prod_LOR_eigs           src/MatrixProductStates.jl:246-253
  * A_prod_L_OO_R_eigs        src/MatrixProductStates.jl:260-266
  * ground_state_search!      src/groundstate.jl:67-147
  * steady_state_search!      src/steadystate.jl:6-86
The reference solves each local eigenproblem with ARPACK `eigs(nev=1, which=:SR, v0, tol)`
(Arpack.jl, not vendored, version unpinned in REQUIRE).  Its published algorithm for one
Hermitian eigenpair is Lanczos; this restatement uses Lanczos with full reorthogonalisation
(twice-applied classical Gram-Schmidt), restarted from the Ritz vector every KMAX steps, the
tridiagonal solved exactly (numpy.linalg.eigh), ARPACK's stopping rule |beta_k s_k| <=
tol |theta|, and the eigenvector's (ARPACK-arbitrary) phase fixed by <v0|x> > 0.
"""
import numpy as np

from .mps_ref import CT, julia_qr, update_le_full, update_re_full

KMAX = 64


def A_prod_LOR_eigs(L, Ain, O, R):
    """out[a0,s,b0] = sum L[a,w,a0] A[a,s',b] O[w,s,w',s'] R[b,w',b0] (L used as stored)."""
    A = np.reshape(Ain, (L.shape[0], O.shape[3], R.shape[0]), order="F")
    out = np.einsum("awx,atb,wsvt,bvy->xsy", L, A, O, R, optimize=True)
    return out.ravel(order="F")


def A_prod_L_OO_R_eigs(L, Ain, O1, O2, R):
    """out = sum L[a,w1,w2,a0] A[a,s,b] O1[w1,t,w1',s] O2[w2,u,w2',t] R[b,w1',w2',b0]."""
    A = np.reshape(Ain, (L.shape[0], O1.shape[3], R.shape[0]), order="F")
    out = np.einsum("apqx,asb,ptvs,qurt,bvry->xuy", L, A, O1, O2, R, optimize=True)
    return out.ravel(order="F")


def lanczos_lowest(matvec, x0, tol, maxiter=1000, kmax=KMAX):
    n = x0.size
    x = np.array(x0, dtype=CT, copy=True)
    iters = 0
    while True:
        nrm = np.linalg.norm(x)
        if nrm == 0.0:
            x = np.zeros(n, dtype=CT)
            x[0] = 1.0
            nrm = 1.0
        V = [x / nrm]
        al, be = [], []
        done = False
        while True:
            w = matvec(V[-1])
            iters += 1
            Vm = np.stack(V, axis=1)
            h = Vm.conj().T @ w
            w = w - Vm @ h
            h2 = Vm.conj().T @ w
            w = w - Vm @ h2
            al.append(h[-1].real + h2[-1].real)
            beta = np.linalg.norm(w)
            T = np.diag(al) + np.diag(be, 1) + np.diag(be, -1)
            ev, evec = np.linalg.eigh(T)
            theta, s = ev[0], evec[:, 0]
            k = len(al) - 1
            conv = abs(beta * s[k]) <= tol * max(abs(theta), 1e-300) or beta <= 1e-14 * (abs(theta) + 1e-300)
            if conv or k + 1 >= n:
                done = True
            if done or iters >= maxiter or k + 1 >= kmax:
                break
            be.append(beta)
            V.append(w / beta)
        if s[0] < 0:
            s = -s
        x = Vm @ s
        if done or iters >= maxiter:
            return theta, x


def ground_state_search_(At, H, maxsweeps, converge_rat, eigs_tol):
    """src/groundstate.jl:67-147 (At updated in place; returns the last eigenvalue)."""
    na = len(At)
    FL, FR = [None] * na, [None] * na
    FL[0] = np.ones((1, 1, 1), dtype=CT)
    for jj in range(na - 1):
        FL[jj + 1] = update_le_full(At[jj], H[jj], At[jj], FL[jj])
    FR[na - 1] = np.ones((1, 1, 1), dtype=CT)
    ae = aestart = 0.0

    def solve(jj):
        return lanczos_lowest(lambda x: A_prod_LOR_eigs(FL[jj], x, H[jj], FR[jj]),
                              At[jj].ravel(order="F"), eigs_tol)

    for _ in range(maxsweeps):
        for jj in range(na - 1, 0, -1):
            ae, av = solve(jj)
            if jj == na - 1:
                aestart = ae
            Dl, d, Dr = At[jj].shape
            q, r = julia_qr(np.reshape(av, (Dl, d * Dr), order="F").conj().T)
            At[jj] = np.reshape(q.conj().T, (q.shape[1], d, Dr), order="F")
            FR[jj - 1] = update_re_full(At[jj], H[jj], At[jj], FR[jj])
            At[jj - 1] = np.einsum("asb,cb->asc", At[jj - 1], r)
        for jj in range(na - 1):
            ae, av = solve(jj)
            Dl, d, Dr = At[jj].shape
            q, r = julia_qr(np.reshape(av, (Dl * d, Dr), order="F"))
            At[jj] = np.reshape(q, (Dl, d, q.shape[1]), order="F")
            FL[jj + 1] = update_le_full(At[jj], H[jj], At[jj], FL[jj])
            At[jj + 1] = np.einsum("cb,bse->cse", r, At[jj + 1])
        ae, av = solve(na - 1)
        At[na - 1] = np.reshape(av, At[na - 1].shape, order="F")
        if abs(ae) > converge_rat * abs(aestart) or abs(ae) < 1e-10:
            break
    return ae


def product_mpo(O2, O1):
    """MPO sites of O2 * O1 (O1 applied first), fused bond index w1 + W1 * w2."""
    out = []
    for a, b in zip(O1, O2):
        p = np.einsum("atbs,cudt->acubds", a, b)
        out.append(np.reshape(p, (a.shape[0] * b.shape[0], b.shape[1], a.shape[2] * b.shape[2], a.shape[3]),
                              order="F"))
    return out


def steady_state_search_(At, L, Lconj, maxsweeps, converge_rat, eigs_tol):
    """src/steadystate.jl:6-86.  Its 4-index environments (update_lenv_two_op / update_renv_two_op)
    and A_prod_L_OO_R_eigs are the 3-index ones of the product MPO Lconj * L with the two bonds
    fused (pinned in tests/test_oracle.py), so this is ground_state_search! on that MPO."""
    return ground_state_search_(At, product_mpo(Lconj, L), maxsweeps, converge_rat, eigs_tol)
