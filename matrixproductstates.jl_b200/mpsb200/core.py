"""Host-side mirror of the MatrixProductStates.jl API for the RK4 path, over the C ABI.

Names follow the reference; Julia's in-place ``f!`` becomes ``f_`` here.  Site indices in
the C ABI are 1-based like Julia; Python lists of sites are 0-based.  Host tensors are
NumPy complex128 arrays in the reference's index order (``A[chiL, d, chiR]``,
``O[wL, d_out, wR, d_in]``) and are moved to / from the device in column-major order.

All compute runs in libmpsb200.so on the GPU; nothing here falls back to the CPU.
"""
import ctypes as C

import numpy as np

from . import _lib

CT = np.complex128


def _f64(arr):
    """Column-major interleaved (re, im) doubles of a complex tensor (a contiguous copy)."""
    a = np.asarray(arr, dtype=CT).ravel(order="F")
    return np.ascontiguousarray(a).view(np.float64)


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64(vals):
    return (C.c_int64 * len(vals))(*[int(v) for v in vals])


class Context:
    """One device + stream + scratch (``mpsb_ctx``)."""

    def __init__(self, device=0):
        h = C.c_void_p()
        _lib.call("mpsb_ctx_create", int(device), C.byref(h))
        self.h = h
        self.device = device

    def sync(self):
        _lib.call("mpsb_sync", self.h)

    def set_graphs(self, enable):
        _lib.call("mpsb_ctx_set_graphs", self.h, 1 if enable else 0)

    def set_pipeline(self, enable):
        """Overlap each RK4 stage's environment initialisation with the previous stage's sweep
        on a second stream (default on; identical results)."""
        _lib.call("mpsb_ctx_set_pipeline", self.h, 1 if enable else 0)

    def set_precision(self, slices, min_tiles=64):
        """Contraction precision of the sweeps: 0 = FP64; 3..7 = int8-sliced tensor-core GEMMs
        with that many slices per operand for GEMMs of at least ``min_tiles`` output tiles."""
        _lib.call("mpsb_ctx_set_precision", self.h, int(slices), int(min_tiles))

    def set_batched_split_threshold(self, min_flops):
        """Batched calls: a GEMM takes the int8-sliced path from ``min_flops`` = 8 M N K of one
        copy's problem (default 2^24; the per-bucket choice of ``mpsb200.autotune``)."""
        _lib.call("mpsb_ctx_set_batched_split_threshold", self.h, float(min_flops))

    def set_profiling(self, enable):
        """Bracket every eager launch of the sliced path's tensor-core GEMM kernel with CUDA
        events (read with ``profile_read``)."""
        _lib.call("mpsb_ctx_set_profiling", self.h, 1 if enable else 0)

    def profile_read(self):
        """(milliseconds, launches, int8 ops) of the tensor-core GEMM kernel since the last read."""
        ms, n, ops = C.c_double(), C.c_int64(), C.c_double()
        _lib.call("mpsb_ctx_profile_read", self.h, C.byref(ms), C.byref(n), C.byref(ops))
        return ms.value, n.value, ops.value

    def set_stream(self, stream_ptr):
        _lib.call("mpsb_ctx_set_stream", self.h, C.c_void_p(stream_ptr or 0))

    @property
    def launches(self):
        v = C.c_int64()
        _lib.call("mpsb_ctx_launch_count", self.h, C.byref(v))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            _lib.call("mpsb_ctx_destroy", self.h)
            self.h = None


_default = None


def default_context():
    global _default
    if _default is None:
        _default = Context(0)
    return _default


class MPS:
    """Device MPS (``Vector{Array{T,3}}``) with fixed bond dims.  With ``batch`` (an int) the
    handle holds that many copies of the shape (a batch handle of the batched engine); site
    access without ``copy`` addresses copy 0."""

    def __init__(self, dims, d, ctx=None, batch=None):
        self.ctx = ctx or default_context()
        self.dims = [int(x) for x in dims]
        self.na = len(self.dims) - 1
        self.d = int(d)
        self.batch = 1 if batch is None else int(batch)
        self.batched = batch is not None
        self.parent = None
        h = C.c_void_p()
        if batch is None:
            _lib.call("mpsb_mps_create", self.ctx.h, self.na, self.d, _i64(self.dims), C.byref(h))
        else:
            _lib.call("mpsb_mps_create_batch", self.ctx.h, self.na, self.d, _i64(self.dims), self.batch, C.byref(h))
        self.h = h

    def view(self, copy):
        """A handle on one copy of a batch handle (shares its memory)."""
        v = MPS.__new__(MPS)
        v.ctx, v.dims, v.na, v.d, v.batch, v.batched, v.parent = self.ctx, self.dims, self.na, self.d, 1, False, self
        h = C.c_void_p()
        _lib.call("mpsb_mps_view", self.h, int(copy), C.byref(h))
        v.h = h
        return v

    def set_site_copy(self, copy, k, a):
        if tuple(a.shape) != self.shape(k):
            raise _lib.DimensionMismatch(-2, "set_site", "site %d has shape %s, expected %s" % (k, a.shape, self.shape(k)))
        buf = _f64(a)
        _lib.call("mpsb_mps_set_site_copy", self.h, int(copy), k + 1, _dptr(buf))

    def site_copy(self, copy, k):
        n = int(np.prod(self.shape(k)))
        buf = np.empty(2 * n, dtype=np.float64)
        _lib.call("mpsb_mps_get_site_copy", self.h, int(copy), k + 1, _dptr(buf))
        return buf.view(CT).reshape(self.shape(k), order="F")

    def sites_copy(self, copy):
        return [self.site_copy(copy, k) for k in range(self.na)]

    def select(self, sources, which):
        """copy b <- sources[which[b]] copy b (which[b] < 0 keeps copy b)."""
        arr = (C.c_void_p * len(sources))(*[s.h.value for s in sources])
        w = (C.c_int * self.batch)(*[int(x) for x in which])
        _lib.call("mpsb_mps_select", self.h, arr, len(sources), w)

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                _lib.call("mpsb_mps_destroy", self.h)
                self.h = None
        except Exception:
            pass

    def __len__(self):
        return self.na

    def shape(self, k):
        return (self.dims[k], self.d, self.dims[k + 1])

    @classmethod
    def from_sites(cls, sites, ctx=None):
        dims = [1] + [int(a.shape[2]) for a in sites]
        m = cls(dims, sites[0].shape[1], ctx)
        m.set_sites(sites)
        return m

    def set_sites(self, sites):
        for k, a in enumerate(sites):
            self.set_site(k, a)

    def set_site(self, k, a):
        if tuple(a.shape) != self.shape(k):
            raise _lib.DimensionMismatch(-2, "set_site", "site %d has shape %s, expected %s" % (k, a.shape, self.shape(k)))
        buf = _f64(a)
        _lib.call("mpsb_mps_set_site", self.h, k + 1, _dptr(buf))

    def site(self, k):
        n = int(np.prod(self.shape(k)))
        buf = np.empty(2 * n, dtype=np.float64)
        _lib.call("mpsb_mps_get_site", self.h, k + 1, _dptr(buf))
        return buf.view(CT).reshape(self.shape(k), order="F")

    def sites(self):
        return [self.site(k) for k in range(self.na)]

    def site_ptr(self, k):
        p = C.c_void_p()
        _lib.call("mpsb_mps_site_ptr", self.h, k + 1, C.byref(p))
        return p.value

    def copy_from(self, other):
        """``self .= copy.(other)``"""
        _lib.call("mpsb_mps_copy", self.h, other.h)
        return self

    def clone(self):
        return MPS(self.dims, self.d, self.ctx, self.batch if self.batched else None).copy_from(self)


class MPO:
    """Device MPO (``Vector{Array{T,4}}``), layout O[wL, d_out, wR, d_in]."""

    def __init__(self, w, d, ctx=None):
        self.ctx = ctx or default_context()
        self.w = [int(x) for x in w]
        self.na = len(self.w) - 1
        self.d = int(d)
        h = C.c_void_p()
        _lib.call("mpsb_mpo_create", self.ctx.h, self.na, self.d, _i64(self.w), C.byref(h))
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                _lib.call("mpsb_mpo_destroy", self.h)
                self.h = None
        except Exception:
            pass

    def __len__(self):
        return self.na

    @classmethod
    def from_sites(cls, sites, ctx=None):
        w = [1] + [int(o.shape[2]) for o in sites]
        m = cls(w, sites[0].shape[1], ctx)
        m.set_sites(sites)
        return m

    def set_sites(self, sites):
        for k, o in enumerate(sites):
            self.set_site(k, o)

    def set_site(self, k, o):
        shp = (self.w[k], self.d, self.w[k + 1], self.d)
        if tuple(o.shape) != shp:
            raise _lib.DimensionMismatch(-2, "set_site", "MPO site %d has shape %s, expected %s" % (k, o.shape, shp))
        buf = _f64(o)
        _lib.call("mpsb_mpo_set_site", self.h, k + 1, _dptr(buf))

    def site(self, k):
        shp = (self.w[k], self.d, self.w[k + 1], self.d)
        buf = np.empty(2 * int(np.prod(shp)), dtype=np.float64)
        _lib.call("mpsb_mpo_get_site", self.h, k + 1, _dptr(buf))
        return buf.view(CT).reshape(shp, order="F")


class Env:
    """``build_env`` buffers (src/constructors.jl:347-375): N+1 entries, ones at both ends."""

    def __init__(self, dims1, dims2, mpo_dims=None, ctx=None, batch=None):
        self.ctx = ctx or default_context()
        self.na = len(dims1) - 1
        self.three = mpo_dims is not None
        self.dims1, self.dims2 = list(dims1), list(dims2)
        self.w = list(mpo_dims) if mpo_dims is not None else [1] * (self.na + 1)
        self.batch = 1 if batch is None else int(batch)
        h = C.c_void_p()
        if batch is None:
            _lib.call("mpsb_env_create", self.ctx.h, self.na, _i64(dims1), _i64(dims2),
                      _i64(self.w) if self.three else None, C.byref(h))
        else:
            _lib.call("mpsb_env_create_batch", self.ctx.h, self.na, _i64(dims1), _i64(dims2),
                      _i64(self.w) if self.three else None, self.batch, C.byref(h))
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                _lib.call("mpsb_env_destroy", self.h)
                self.h = None
        except Exception:
            pass

    def entry_shape(self, e):
        end = e == 0 or e == self.na
        a = 1 if end else self.dims1[e]
        b = 1 if end else self.dims2[e]
        w = 1 if end else int(self.w[e])
        return (a, w, b) if self.three else (a, b)

    def entry(self, e):
        shp = self.entry_shape(e)
        buf = np.empty(2 * int(np.prod(shp)), dtype=np.float64)
        _lib.call("mpsb_env_get", self.h, e + 1, _dptr(buf))
        return buf.view(CT).reshape(shp, order="F")

    def set_entry(self, e, x):
        buf = _f64(x)
        _lib.call("mpsb_env_set", self.h, e + 1, _dptr(buf))


def build_env(dims1, dims2, mpo_dims=None, ctx=None, batch=None):
    return Env(dims1, dims2, mpo_dims, ctx, batch)


# ------------------------------------------------------------------ constructors

def _dims_rule(na, dmax, d):
    dims = [1] * (na + 1)
    for k in range(1, na):
        dims[k] = dmax
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
    return dims


def mpsproductstate(na, dmax, d, state, ctx=None):
    """src/constructors.jl:8-61: padded product state, left-orthogonalised on the GPU with R
    carried right (the same QR sweep as leftorthogonalizeQR!)."""
    st = state if callable(state) else (lambda n: state)
    dims = _dims_rule(na, dmax, d)
    mps = MPS(dims, d, ctx)
    for n in range(1, na + 1):
        site = np.zeros((dims[n - 1], d, dims[n]), dtype=CT)
        site[0, :, 0] = np.asarray(st(n), dtype=CT)
        mps.set_site(n - 1, site)
    leftorthogonalizeQR_(mps)
    return mps, dims


def mpsgroundstate(na, dmax, d, ctx=None):
    """src/constructors.jl:69-75."""
    state = np.zeros(d, dtype=CT)
    state[0] = 1.0
    return mpsproductstate(na, dmax, d, state, ctx)


def mpsrandom(na, dmax, d, rng, ctx=None):
    """src/constructors.jl:113-129 with i.i.d. complex Gaussian sites (SQRT_HALF*(re + i im),
    src/MatrixProductStates.jl:24-27) drawn from ``rng`` in memory order, each site then
    replaced by the Q of its own QR (leftorth!) on the GPU."""
    dims = _dims_rule(na, dmax, d)
    mps = MPS(dims, d, ctx)
    s = np.sqrt(0.5)
    for n in range(na):
        shape = (dims[n], d, dims[n + 1])
        k = int(np.prod(shape))
        flat = (s * rng.standard_normal(k) + 1j * s * rng.standard_normal(k)).astype(CT)
        mps.set_site(n, flat.reshape(shape, order="F"))
    leftorth_sites_(mps)
    return mps, dims


def leftorth_sites_(mps):
    """``mps[n] = leftorth!(mps[n])`` for every site (Q only, no R carried)."""
    for n in range(mps.na):
        Dl, d, Dr = mps.shape(n)
        p = mps.site_ptr(n)
        _lib.call("mpsb_op_qr", mps.ctx.h, C.c_void_p(p), C.c_void_p(p), None, Dl * d, Dr)


def expandmps(mps, dmax, ctx=None):
    """src/constructors.jl:134-162: zero-pad to bond dim dmax, then left-orthogonalise."""
    na, d = mps.na, mps.d
    dims = [dmax] * (na + 1)
    dims[0] = dims[na] = 1
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
    out = MPS(dims, d, ctx or mps.ctx)
    for n in range(na):
        a = mps.site(n)
        site = np.zeros((dims[n], d, dims[n + 1]), dtype=CT)
        site[: a.shape[0], :, : a.shape[2]] = a
        out.set_site(n, site)
    leftorthogonalizeQR_(out)
    return out, dims


def makempo(mpomat, na, d, ctx=None):
    """src/constructors.jl:231-253: ``mpomat[l][m]`` a callable of the 1-based site."""
    b1, b2 = len(mpomat), len(mpomat[0])
    sites = []
    for n in range(1, na + 1):
        o = np.zeros((b1, d, b2, d), dtype=CT)
        for m in range(b2):
            for l in range(b1):
                o[l, :, m, :] = np.asarray(mpomat[l][m](n), dtype=CT) * np.ones((d, d))
        sites.append(o)
    sites[0] = sites[0][0:1].copy()
    sites[-1] = sites[-1][:, :, b2 - 1:b2].copy()
    return MPO.from_sites(sites, ctx)


def makemps(mpsmat, na, d, ctx=None):
    """src/constructors.jl:200-222."""
    b1, b2 = len(mpsmat), len(mpsmat[0])
    sites = []
    for n in range(1, na + 1):
        a = np.zeros((b1, d, b2), dtype=CT)
        for m in range(b2):
            for l in range(b1):
                a[l, :, m] = np.asarray(mpsmat[l][m](n), dtype=CT)
        sites.append(a)
    sites[0] = sites[0][0:1].copy()
    sites[-1] = sites[-1][:, :, b2 - 1:b2].copy()
    return MPS.from_sites(sites, ctx)


# ------------------------------------------------------------------ hot path

def RK4stp_apply_H_half_(dt, H, *args):
    """``RK4stp_apply_H_half!`` (src/timeevolution.jl:178-196).

    10-argument form ``(dt, H, psi, psi1, psi2, psi3, env1, env2, env3, envop)`` updates psi
    in place; 11-argument form ``(dt, H, psi0, psi, psi1, ...)`` writes psi0."""
    if len(args) == 8:
        psi, psi1, psi2, psi3, env1, env2, env3, envop = args
        psi0 = psi
    elif len(args) == 9:
        psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop = args
    else:
        raise TypeError("RK4stp_apply_H_half_ takes 10 or 11 arguments")
    ctx = psi.ctx
    _lib.call("mpsb_rk4stp_apply_H_half", ctx.h, float(dt), H[0].h, H[1].h, H[2].h, psi0.h, psi.h,
              psi1.h, psi2.h, psi3.h, env1.h, env2.h, env3.h, envop.h)


def compress_var_apply_H_left_(A0, envop, Ain, A, H):
    """src/compression.jl:321-347."""
    _lib.call("mpsb_compress_var_apply_H_left", A0.ctx.h, A0.h, envop.h, Ain.h, A.h, H.h)


def _coef_buf(coef):
    c = np.asarray(coef, dtype=CT)
    return np.ascontiguousarray(c).view(np.float64)


def _sum_var(name, A0, env, envop, Ain, coef, A, H):
    numv = len(coef)
    if len(A) != numv or len(env) != numv - 1:
        raise _lib.DimensionMismatch(-2, name, "len(A) must be len(coef), len(env) len(coef)-1")
    cb = _coef_buf(coef)
    envs = (C.c_void_p * max(1, len(env)))(*[e.h.value for e in env])
    terms = (C.c_void_p * numv)(*[a.h.value for a in A])
    _lib.call(name, A0.ctx.h, A0.h, envs, envop.h, Ain.h, _dptr(cb), numv, terms, H.h)


def compress_sum_var_apply_H_right_(A0, env, envop, Ain, coef, A, H):
    """src/compression.jl:1007-1063."""
    _sum_var("mpsb_compress_sum_var_apply_H_right", A0, env, envop, Ain, coef, A, H)


def compress_sum_var_apply_H_left_(A0, env, envop, Ain, coef, A, H):
    """src/compression.jl:889-944."""
    _sum_var("mpsb_compress_sum_var_apply_H_left", A0, env, envop, Ain, coef, A, H)


def compress_var_apply_H_(A0, envop, Ain, A, H, maxsweeps):
    """src/compression.jl:217-258."""
    _lib.call("mpsb_compress_var_apply_H", A0.ctx.h, A0.h, envop.h, Ain.h, A.h, H.h, int(maxsweeps))


def _terms(name, coef, A):
    numv = len(coef)
    if len(A) != numv:
        raise _lib.DimensionMismatch(-2, name, "len(A) must be len(coef)")
    return numv, _coef_buf(coef), (C.c_void_p * numv)(*[a.h.value for a in A])


def compress_sum_var_apply_H_(A0, envop, coef, A, H, maxsweeps):
    """src/compression.jl:805-887: A0 (guess and output) <- the variational compression of
    sum_l coef[l] A[l] + coef[-1] H A[-1] with maxsweeps sweep pairs."""
    numv, cb, terms = _terms("compress_sum_var_apply_H!", coef, A)
    _lib.call("mpsb_compress_sum_var_apply_H", A0.ctx.h, A0.h, envop.h, _dptr(cb), numv, terms, H.h, int(maxsweeps))


def compress_sum_var(Ain, coef, A, maxsweeps):
    """src/compression.jl:496-565: a new MPS compressing sum_l coef[l] A[l], guess Ain."""
    numv, cb, terms = _terms("compress_sum_var", coef, A)
    A0 = MPS(Ain.dims, Ain.d, Ain.ctx)
    _lib.call("mpsb_compress_sum_var", A0.ctx.h, A0.h, Ain.h, _dptr(cb), numv, terms, int(maxsweeps))
    return A0


def Arnoldi_expm_(A, rhov, numv, env, envop):
    """src/timeevolution.jl:88-119: Krylov step rhov[0] <- exp(A) rhov[0] (normalised) in the
    span of numv MPSs built by repeated application of the MPO A (one sweep pair each, then
    normalize_lo!), with the projected generator H and overlap matrix N measured by
    scal_op_prod / scal_prod and coef = expm(N \\ H)[:, 0].  `env` is unused, as in the
    reference (the plain-term environments are internal).  rhov[0] is rebound to a new MPS."""
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
    rhov[0] = compress_sum_var(rhov[0], list(coef), rhov, 1)
    normalize_lo_(rhov[0])
    return coef


def ground_state_search_(At, H, maxsweeps, converge_rat, eigs_tol):
    """src/groundstate.jl:67-147: At (left canonical guess) <- single-site ground-state sweeps
    of the MPO H; returns the last local eigenvalue."""
    ae = C.c_double()
    _lib.call("mpsb_ground_state_search", At.ctx.h, At.h, H.h, int(maxsweeps), float(converge_rat),
              float(eigs_tol), C.byref(ae))
    return ae.value


def product_mpo(O2, O1, ctx=None):
    """The MPO of O2 * O1 (O1 applied first), fused bond index w1 + W1 * w2: the operator that
    A_prod_L_OO_R_eigs (src/MatrixProductStates.jl:260-266) applies with O1 = L, O2 = Lconj."""
    sites = []
    for k in range(O1.na):
        a, b = O1.site(k), O2.site(k)   # [w, d_out, w', d_in]
        p = np.einsum("atbs,cudt->acubds", a, b)
        w1, w2, dd, w1p, w2p = a.shape[0], b.shape[0], b.shape[1], a.shape[2], b.shape[2]
        sites.append(p.reshape((w1 * w2, dd, w1p * w2p, a.shape[3]), order="F"))
    return MPO.from_sites(sites, ctx or O1.ctx)


def steady_state_search_(At, L, Lconj, maxsweeps, converge_rat, eigs_tol):
    """src/steadystate.jl:6-86: ground_state_search! with the effective operator Lconj * L
    (A_prod_L_OO_R_eigs with 4-index environments is the same contraction with the two MPO
    bonds fused)."""
    return ground_state_search_(At, product_mpo(Lconj, L, At.ctx), maxsweeps, converge_rat, eigs_tol)


def compressionSVD_(mps, dmax, tol=1e-15):
    """src/compression.jl:1280-1312: right-to-left SVD truncation of the left-canonical mps to
    bond dims <= dmax with relative weight tolerance tol.  The reference resizes mps in place;
    a handle cannot change its dims, so the truncated (right-canonical) MPS is returned first:
    (new_mps, err_glob, err_trim, ent_ent)."""
    out = C.c_void_p()
    eg = C.c_double()
    et = np.zeros(mps.na)
    ee = np.zeros(mps.na)
    _lib.call("mpsb_compression_svd", mps.ctx.h, mps.h, int(dmax), float(tol), C.byref(out), C.byref(eg),
              _dptr(et), _dptr(ee))
    return _wrap_new_mps(out, mps.ctx, mps.na, mps.d), eg.value, et, ee


def _wrap_new_mps(h, ctx, na, d):
    new = MPS.__new__(MPS)
    new.ctx, new.na, new.d, new.h = ctx, na, d, h
    info = np.zeros(na + 1, dtype=np.int64)
    _lib.call("mpsb_mps_info", h, None, None, info.ctypes.data_as(C.POINTER(C.c_int64)))
    new.dims = [int(x) for x in info]
    return new


def compress_var_apply_H_two_site(Ain, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:355-411: two-site variational compression of H*A with SVD truncation
    (bonds adapt up to dlim).  Returns the new MPS; `dims` (a list) is updated in place like
    the reference's."""
    out = C.c_void_p()
    _lib.call("mpsb_compress_var_apply_H_two_site", Ain.ctx.h, Ain.h, A.h, H.h, int(maxsweeps), float(svd_tol),
              int(dlim), C.byref(out))
    new = _wrap_new_mps(out, Ain.ctx, Ain.na, Ain.d)
    dims[:] = new.dims
    return new


def compress_var_two_site(Ain, A, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:110-165: the same compression of A itself (an identity operator)."""
    ident = np.eye(A.d, dtype=CT).reshape(1, A.d, 1, A.d)
    Id = MPO.from_sites([ident] * A.na, A.ctx)
    return compress_var_apply_H_two_site(Ain, A, Id, maxsweeps, svd_tol, dims, dlim)


# The reference's allocating forms: a new output MPS (the guess's dims) and internal
# environments around the in-place entry points above.

def compress_var(Ain, A, maxsweeps):
    """src/compression.jl:19-62: a new MPS, the variational compression of A (guess Ain)."""
    return compress_sum_var(Ain, [1.0], [A], maxsweeps)


def _new_like(Ain, H=None, plain=0):
    A0 = Ain.clone()
    envop = build_env(Ain.dims, Ain.dims, H.w, Ain.ctx) if H is not None else None
    env = [build_env(Ain.dims, Ain.dims, None, Ain.ctx) for _ in range(plain)]
    return A0, envop, env


def compress_var_apply_H(Ain, A, H, maxsweeps):
    """src/compression.jl:173-215: a new MPS compressing H*A with maxsweeps sweep pairs."""
    A0, envop, _ = _new_like(Ain, H)
    compress_var_apply_H_(A0, envop, Ain, A, H, maxsweeps)
    return A0


def compress_var_apply_H_left(Ain, A, H):
    """src/compression.jl:291-319: one right-to-left sweep of H*A from left environments of Ain."""
    A0, envop, _ = _new_like(Ain, H)
    compress_var_apply_H_left_(A0, envop, Ain, A, H)
    return A0


def compress_var_apply_H_right(Ain, A, H, maxsweeps=1):
    """src/compression.jl:261-289: one left-to-right sweep of H*A from right environments of Ain
    (maxsweeps is unused, as in the reference)."""
    A0, envop, _ = _new_like(Ain, H)
    compress_sum_var_apply_H_right_(A0, [], envop, Ain, [1.0], [A], H)
    return A0


def compress_sum_var_apply_H(Ain, coef, A, H, maxsweeps):
    """src/compression.jl:657-740: a new MPS compressing sum_l coef[l] A[l] + coef[-1] H A[-1]."""
    A0, envop, _ = _new_like(Ain, H)
    compress_sum_var_apply_H_(A0, envop, coef, A, H, maxsweeps)
    return A0


def compress_sum_var_apply_H_left(Ain, coef, A, H):
    """src/compression.jl:742-802: one right-to-left sweep (coefficients on the right boundary)."""
    A0, envop, env = _new_like(Ain, H, len(coef) - 1)
    compress_sum_var_apply_H_left_(A0, env, envop, Ain, coef, A, H)
    return A0


def compress_sum_var_apply_H_right(Ain, coef, A, H):
    """src/compression.jl:946-1005: one left-to-right sweep (coefficients on the left boundary)."""
    A0, envop, env = _new_like(Ain, H, len(coef) - 1)
    compress_sum_var_apply_H_right_(A0, env, envop, Ain, coef, A, H)
    return A0


def _sum_two_site(name, Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim, half):
    numv, cb, terms = _terms(name, coef, A)
    out = C.c_void_p()
    _lib.call("mpsb_compress_sum_var_apply_H_two_site", Ain.ctx.h, Ain.h, _dptr(cb), numv, terms,
              H.h if H is not None else None, int(maxsweeps), float(svd_tol), int(dlim), int(half), C.byref(out))
    new = _wrap_new_mps(out, Ain.ctx, Ain.na, Ain.d)
    dims[:] = new.dims
    return new


def compress_sum_var_apply_H_two_site(Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:1072-1157: two-site variational compression of
    sum_l coef[l] A[l] + coef[-1] H A[-1] (guess Ain, left canonical).  Returns the new MPS;
    `dims` is updated in place."""
    return _sum_two_site("compress_sum_var_apply_H_two_site", Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim, 0)


def compress_sum_var_apply_H_two_site_left(Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:1159-1215: one right-to-left two-site sweep (first site U diag(S))."""
    return _sum_two_site("compress_sum_var_apply_H_two_site_left", Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim, 1)


def compress_sum_var_apply_H_two_site_right(Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:1218-1276: one left-to-right two-site sweep from a right-canonical
    guess (coefficients on the left boundary; last site diag(S) V')."""
    return _sum_two_site("compress_sum_var_apply_H_two_site_right", Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim, 2)


def compress_var_apply_H_two_site_left(Ain, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:413-448: one right-to-left two-site sweep of H*A (first site U diag(S))."""
    return compress_sum_var_apply_H_two_site_left(Ain, [1.0], [A], H, maxsweeps, svd_tol, dims, dlim)


def compress_var_apply_H_two_site_right(Ain, A, H, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:450-486: one left-to-right two-site sweep of H*A from a right-canonical
    guess (last site diag(S) V')."""
    return compress_sum_var_apply_H_two_site_right(Ain, [1.0], [A], H, maxsweeps, svd_tol, dims, dlim)


def RK4stp_apply_H_half_full_two_site(dt, H, psi, svd_tol, dims, dlim):
    """src/timeevolution.jl:208-215: the RK4 step with every stage a two-site half sweep
    (R->L, L->R, R->L, L->R), so the bond dims adapt to the state (<= dlim, truncation rule of
    compressionSVD! with svd_tol); `dims` is updated in place and the new psi returned."""
    psi1 = compress_var_apply_H_two_site_left(psi, psi, H[0], 1, svd_tol, dims, dlim)
    psi2 = compress_sum_var_apply_H_two_site_right(psi1, [1.0, dt / 2], [psi, psi1], H[1], 1, svd_tol, dims, dlim)
    psi3 = compress_sum_var_apply_H_two_site_left(psi2, [1.0, dt], [psi, psi2], H[1], 1, svd_tol, dims, dlim)
    return compress_sum_var_apply_H_two_site_right(psi3, [-1 / 3, 1 / 3, 2 / 3, 1 / 3], [psi, psi1, psi2, psi3], H[2],
                                                   1, svd_tol, dims, dlim)


def compress_sum_var_two_site(Ain, coef, A, maxsweeps, svd_tol, dims, dlim):
    """src/compression.jl:574-648: the same with every term plain (no operator)."""
    return _sum_two_site("compress_sum_var_two_site", Ain, coef, A, None, maxsweeps, svd_tol, dims, dlim, 0)


# ------------------------------------------------------------------ norms, gauge, observables

def _scalar(name, *args):
    v = C.c_double()
    _lib.call(name, *args, C.byref(v))
    return v.value


def normalize_lo_(mps):
    """src/orthonormalisation.jl:97-103."""
    return _scalar("mpsb_normalize_lo", mps.ctx.h, mps.h)


def normalize_lo_batch(mps, allow_nonfinite=False):
    """normalize_lo! of every copy of a batch handle; returns the norms^2 before scaling.  A copy
    whose norm is NaN or infinite raises MPSB_ERR_NONFINITE, unless allow_nonfinite, which returns
    the norms as they are (the caller checks each copy)."""
    out = np.zeros(mps.batch, dtype=np.float64)
    try:
        _lib.call("mpsb_normalize_lo_batch", mps.ctx.h, mps.h, _dptr(out))
    except _lib.MpsbError as e:
        if not (allow_nonfinite and e.status == -6):
            raise
    return out


def norm_lo(mps):
    """src/orthonormalisation.jl:117-121."""
    return _scalar("mpsb_norm_lo", mps.ctx.h, mps.h)


def leftorthonormalizationQR_(mps):
    """src/orthonormalisation.jl:29-36."""
    return _scalar("mpsb_leftorthonormalizationQR", mps.ctx.h, mps.h)


def leftorthogonalizeQR_(mps):
    """src/orthonormalisation.jl:43-56."""
    return _scalar("mpsb_leftorthogonalizeQR", mps.ctx.h, mps.h)


def apply_site_operator_(mps, site, op):
    """src/MatrixProductStates.jl:135-143 on ``mps[site]`` (1-based site like the reference)."""
    buf = _f64(np.asarray(op, dtype=CT))
    _lib.call("mpsb_apply_site_operator", mps.ctx.h, mps.h, int(site), _dptr(buf))


def _complex(name, *args):
    out = np.zeros(2, dtype=np.float64)
    _lib.call(name, *args, _dptr(out))
    return complex(out[0], out[1])


def scal_prod(mps1, mps2):
    """src/MatrixProductStates.jl:345-358."""
    return _complex("mpsb_scal_prod", mps1.ctx.h, mps1.h, mps2.h)


def scal_op_prod(mps1, op, mps2):
    """src/MatrixProductStates.jl:327-340."""
    return _complex("mpsb_scal_op_prod", mps1.ctx.h, mps1.h, op.h, mps2.h)


def scal_prod_no_conj(mps1, mps2):
    """src/MatrixProductStates.jl:366-379."""
    return _complex("mpsb_scal_prod_no_conj", mps1.ctx.h, mps1.h, mps2.h)


def measure_local(mps, op):
    """Local <op_n> for every site of a left-orthonormal MPS: the right-to-left local_exp sweep
    of measure_excitations! (examples/spin_model_quantum_trajectory_rk4.jl:220-231)."""
    out = np.zeros(mps.na, dtype=np.float64)
    buf = _f64(np.asarray(op, dtype=CT))
    _lib.call("mpsb_measure_local", mps.ctx.h, mps.h, _dptr(buf), _dptr(out))
    return out


def applyMPOtoMPS(mps, mpo):
    """src/MatrixProductStates.jl:115-133 (exact; bond dims multiply)."""
    dims = [a * w for a, w in zip(mps.dims, mpo.w)]
    out = MPS(dims, mps.d, mps.ctx)
    _lib.call("mpsb_apply_mpo_to_mps", mps.ctx.h, mps.h, mpo.h, out.h)
    return out
