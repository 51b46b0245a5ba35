"""Batched quantum trajectories: many independent trajectories of one chain in one engine.

The reference runs one trajectory per process (examples/spin_model_quantum_trajectory_rk4.jl:
104-209, one seed per run).  Here trajectories whose bond-dim cap is the same share a bucket:
the bucket's states live in batch handles (all copies of one MPS shape back to back), and every
step of the example loop is issued once for the whole bucket --

  * the coherent RK4 step (RK4stp_apply_H_half!) of every copy, one captured CUDA graph whose
    GEMM, MPO-apply and cluster-QR launches each cover all copies;
  * normalize_lo! of A_coh for every copy, one read-back of the norms;
  * on a step where some copy jumps (r1 >= p_coh), the two waveguide-jump compressions
    compress_var_apply_H!(A_r / A_l, ..., jumpright / jumpleft, 1) and their normalize_lo! for
    every copy of the bucket (the reference computes them only on its jump steps; computing them
    for the bucket's other copies as well changes nothing for those and keeps the launches
    batched);
  * the host decision of each trajectory with its own r1 / r2 stream (the example's branch
    logic), then one per-copy select A <- A_coh / A_r / A_l; local decays (gam_eg > 0) act on a
    view of the copy.

Buckets run on their own contexts (streams), so the buckets' kernels overlap on the device.
Within a bucket every kernel computes each copy exactly as it computes a bucket of one (batched
calls choose every kernel's partition from one copy's shape), so a trajectory's records and
state do not depend on which other trajectories share its bucket.
"""
import numpy as np

from . import autotune as AT
from . import core as K
from . import models as Mo


def dims_rule(na, dmax, d):
    dims = [dmax] * (na + 1)
    dims[0] = dims[na] = 1
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
    return dims


class TrajectoryBucket:
    """All trajectories of one bond-dim cap `chi`: the example's buffers as batch handles."""

    def __init__(self, p, chi, dt, r1, r2, device=0, ctx=None, slices=0, tuned=False):
        self.p, self.chi, self.dt = p, int(chi), dt
        # every copy's own uniform streams and step index (copies may start at different steps
        # when a serving loop hands a slot to a new job, see assign)
        self.r1 = [np.asarray(x, dtype=np.float64) for x in np.atleast_2d(r1)]
        self.r2 = [np.asarray(x, dtype=np.float64) for x in np.atleast_2d(r2)]
        self.B = len(self.r1)
        self.t = np.zeros(self.B, dtype=np.int64)
        self.active = np.ones(self.B, dtype=bool)
        self.ctx = ctx or K.Context(device)
        self.own_ctx = ctx is None
        # tuned: the autotuner's (slices, threshold) for this shape (mpsb200.autotune)
        self.slices = AT.apply(self.ctx, "trajectory", 2, 4, self.chi, slices) if tuned else slices
        if not tuned:
            self.ctx.set_precision(slices)
        na = p.na
        dims = dims_rule(na, self.chi, 2)
        self.dims = dims
        B, c = self.B, self.ctx
        self.A = K.MPS(dims, 2, c, batch=B)
        # mpsgroundstate (src/constructors.jl:67-76): the padded product state left-orthogonalised
        # by the QR sweep (its zero-weight columns are the Householder ones), in every copy
        start, _ = K.mpsgroundstate(na, self.chi, 2, c)
        self.start_sites = start.sites()
        for k, site in enumerate(self.start_sites):
            for b in range(B):
                self.A.set_site_copy(b, k, site)
        del start
        self.A_coh, self.A_r, self.A_l, self.A1, self.A2, self.A3 = (K.MPS(dims, 2, c, batch=B) for _ in range(6))
        self.envop = K.build_env(dims, dims, [4] * (na + 1), c, batch=B)
        self.envop_jump = K.build_env(dims, dims, [2] * (na + 1), c, batch=B)
        self.env1, self.env2, self.env3 = (K.build_env(dims, dims, None, c, batch=B) for _ in range(3))
        self.H = [K.MPO.from_sites(Mo.sm_hamiltonian(p, 1, dt / 2, 0.0), c),
                  K.MPO.from_sites(Mo.sm_hamiltonian(p, 0, 1, dt / 2), c),
                  K.MPO.from_sites(Mo.sm_hamiltonian(p, 1, dt / 2, dt), c)]
        jr_, jl_ = Mo.jump_mpos(p, 0.0)
        self.jumpright = K.MPO.from_sites(jr_, c)
        self.jumpleft = K.MPO.from_sites(jl_, c)
        self.p_coh = [[] for _ in range(B)]
        self.jumps = [[] for _ in range(B)]
        self.i = 0

    def refresh_h(self, host_sites):
        """Upload the three generator MPOs of this step from host site arrays (the example loop's
        update_h!, examples/spin_model_quantum_trajectory_rk4.jl:115-118)."""
        for mpo, sites in zip(self.H, host_sites):
            mpo.set_sites(sites)

    def assign(self, b, r1, r2):
        """Give copy b to a new trajectory: the start state, its own uniform streams, step 0."""
        self.reset(b)
        self.r1[b], self.r2[b] = np.asarray(r1, dtype=np.float64), np.asarray(r2, dtype=np.float64)
        self.t[b] = 0
        self.p_coh[b], self.jumps[b] = [], []
        self.active[b] = True

    def release(self, b):
        """Copy b keeps being stepped with the others but carries no trajectory."""
        self.active[b] = False

    def reset(self, b):
        """Copy b <- the start state (a released copy whose state went bad)."""
        for k, site in enumerate(self.start_sites):
            self.A.set_site_copy(b, k, site)

    def state(self, b):
        return self.A.sites_copy(b)

    def issue(self):
        """Enqueue step i's coherent step for every copy (no wait)."""
        K.RK4stp_apply_H_half_(self.dt, self.H, self.A_coh, self.A, self.A1, self.A2, self.A3,
                               self.env1, self.env2, self.env3, self.envop)

    def finish(self, bad=None):
        """Norms, each active trajectory's decision of its own step, and the state update
        A <- chosen copy.  With `bad` (a list), a copy whose norm is not finite is appended to it
        and released instead of raising (a serving loop fails that job alone)."""
        p, dt, na = self.p, self.dt, self.p.na
        p_coh = K.normalize_lo_batch(self.A_coh, allow_nonfinite=bad is not None)
        if bad is not None:
            for b in range(self.B):
                if self.active[b] and not (np.isfinite(p_coh[b]) and p_coh[b] <= 1e300):
                    bad.append(b)
                    self.active[b] = False
        act = [b for b in range(self.B) if self.active[b]]
        p_r = p_l = None
        if any(self.r1[b][self.t[b]] >= p_coh[b] for b in act):   # a jump step for some copy
            K.compress_var_apply_H_(self.A_r, self.envop_jump, self.A, self.A, self.jumpright, 1)
            p_r = K.normalize_lo_batch(self.A_r)
            K.compress_var_apply_H_(self.A_l, self.envop_jump, self.A, self.A, self.jumpleft, 1)
            p_l = K.normalize_lo_batch(self.A_l)
        which = np.zeros(self.B, dtype=np.int64)   # released copies keep their coherent step
        local = []
        for b in act:
            i = int(self.t[b])
            self.t[b] += 1
            self.p_coh[b].append(p_coh[b])
            if self.r1[b][i] < p_coh[b]:
                continue
            p_acc = np.zeros(na + 3)
            if p.gam_eg != 0:
                epop = K.measure_local(self.A.view(b), Mo.E_E)
                for j in range(na):
                    p_acc[j + 1] = p_acc[j] + dt * p.gam_eg * epop[j]
            p_acc[na + 1] = p_acc[na] + dt * p_r[b]
            p_acc[na + 2] = p_acc[na + 1] + dt * p_l[b]
            p_sum = p_acc[-1]
            p_acc = p_acc / p_acc[-1]
            r = self.r2[b][i]
            if r < p_acc[na]:
                which[b] = -1   # the local decay acts on the step's start state
                for j in range(na):
                    if r < p_acc[j + 1]:
                        local.append((b, j))
                        self.jumps[b].append((i, "local", j + 1, p_coh[b], p_sum))
                        break
            elif r < p_acc[na + 1]:
                which[b] = 1
                self.jumps[b].append((i, "right", 0, p_coh[b], p_sum))
            else:
                which[b] = 2
                self.jumps[b].append((i, "left", 0, p_coh[b], p_sum))
        self.A.select([self.A_coh, self.A_r, self.A_l], which)
        for b, j in local:
            v = self.A.view(b)
            K.apply_site_operator_(v, j + 1, Mo.SM)
            K.leftorthonormalizationQR_(v)
        self.i += 1

    def close(self):
        for name in ("A", "A_coh", "A_r", "A_l", "A1", "A2", "A3", "envop", "envop_jump", "env1", "env2", "env3",
                     "H", "jumpright", "jumpleft"):
            setattr(self, name, None)
        if self.own_ctx:
            self.ctx.close()


class DensityBucket:
    """Density-matrix evolutions of one shape (N, chi, w, dt) in the copies of batch handles: the
    in-place RK4 step of examples/spin_model_density_matrix.jl for every copy in one call.  Copies
    are handed to jobs (assign) and given back (release) by a serving loop; each copy counts its
    own steps."""

    def __init__(self, p, chi, dt, B, w=8, device=0, ctx=None, slices=0, tuned=False):
        self.p, self.chi, self.dt, self.B, self.w = p, int(chi), dt, int(B), int(w)
        self.ctx = ctx or K.Context(device)
        self.own_ctx = ctx is None
        self.slices = AT.apply(self.ctx, "density", 4, self.w, self.chi, slices) if tuned else slices
        if not tuned:
            self.ctx.set_precision(slices)
        na, c = p.na, self.ctx
        dims = dims_rule(na, self.chi, 4)
        self.dims = dims
        start, _ = K.mpsgroundstate(na, self.chi, 4, c)
        self.start_sites = start.sites()
        del start
        self.rho, self.rho1, self.rho2, self.rho3 = (K.MPS(dims, 4, c, batch=self.B) for _ in range(4))
        for b in range(self.B):
            self.reset(b)
        self.env1, self.env2, self.env3 = (K.build_env(dims, dims, None, c, batch=self.B) for _ in range(3))
        self.envop = K.build_env(dims, dims, [max(6, self.w)] * (na + 1), c, batch=self.B)
        self.L = [K.MPO.from_sites(Mo.construct_L_spin_model(p, 1, dt / 2, 0.0, self.w), c),
                  K.MPO.from_sites(Mo.construct_L_spin_model(p, 0, 1, dt / 2, self.w), c),
                  K.MPO.from_sites(Mo.construct_L_spin_model(p, 1, dt / 2, dt, self.w), c)]
        self.t = np.zeros(self.B, dtype=np.int64)
        self.active = np.zeros(self.B, dtype=bool)

    def reset(self, b):
        """Copy b <- the all-down product density matrix (mpsgroundstate with d = 4)."""
        for k, site in enumerate(self.start_sites):
            self.rho.set_site_copy(b, k, site)

    def assign(self, b):
        self.reset(b)
        self.t[b] = 0
        self.active[b] = True

    def release(self, b):
        self.active[b] = False

    def issue(self):
        """Enqueue one in-place RK4 step of every copy (no wait)."""
        K.RK4stp_apply_H_half_(self.dt, self.L, self.rho, self.rho1, self.rho2, self.rho3,
                               self.env1, self.env2, self.env3, self.envop)

    def finish(self, bad=None):
        self.t[self.active] += 1

    def state(self, b):
        return self.rho.sites_copy(b)

    def close(self):
        for name in ("rho", "rho1", "rho2", "rho3", "env1", "env2", "env3", "envop", "L"):
            setattr(self, name, None)
        if self.own_ctx:
            self.ctx.close()


class TrajectoryBatch:
    """Trajectories of one chain with per-trajectory bond caps `chis` and uniform streams
    r1[k], r2[k]; grouped into buckets of equal cap; `slices` > 0 puts the sweeps' larger
    contractions on the int8-sliced tensor-core path (see Context.set_precision)."""

    def __init__(self, p, chis, dt, r1, r2, device=0, slices=0, tuned=False):
        self.p, self.dt = p, dt
        self.chis = [int(c) for c in chis]
        r1, r2 = np.asarray(r1), np.asarray(r2)
        self.members = {}
        for k, c in enumerate(self.chis):
            self.members.setdefault(c, []).append(k)
        self.buckets = {c: TrajectoryBucket(p, c, dt, r1[m], r2[m], device, slices=slices, tuned=tuned)
                        for c, m in sorted(self.members.items())}

    def generator_sites(self, t):
        """Host site arrays of the step's three generator MPOs at time t (H[1..3] of the example)."""
        p, dt = self.p, self.dt
        return [Mo.sm_hamiltonian(p, 1, dt / 2, t), Mo.sm_hamiltonian(p, 0, 1, t + dt / 2),
                Mo.sm_hamiltonian(p, 1, dt / 2, t + dt)]

    def step(self, host_h=None):
        """One step of every trajectory; with host_h (generator_sites of the step's time) the
        generators are uploaded first, as the example loop refreshes them every step."""
        for bk in self.buckets.values():
            if host_h is not None:
                bk.refresh_h(host_h)
            bk.issue()
        for bk in self.buckets.values():
            bk.finish()

    def records(self, k):
        """(p_coh, jumps, final sites) of trajectory k."""
        c = self.chis[k]
        b = self.members[c].index(k)
        bk = self.buckets[c]
        return np.array(bk.p_coh[b]), list(bk.jumps[b]), bk.A.sites_copy(b)

    def site_updates_per_step(self):
        return self.p.na * len(self.chis)

    def close(self):
        for bk in self.buckets.values():
            bk.close()
