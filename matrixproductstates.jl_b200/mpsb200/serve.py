"""Serving loop: a stream of trajectory and density-matrix jobs sharing one GPU.

Jobs arrive over time (seeded Poisson arrivals) and are admitted while the number of running
jobs and their device footprint stay inside the limits; a job keeps its MPS state on the device
until it finishes.  Two ways of placing jobs:

* ``mode="shared"`` (the default): continuous batching.  Jobs of the same shape (kind, N, chi,
  dt) share a bucket -- the batch handles of the batched engine (`batch.TrajectoryBucket`,
  `batch.DensityBucket`), whose every RK4 step is one batched call for all its copies.  A job
  takes a free copy ("slot") of a running bucket of its shape as soon as one is free, at whatever
  step the bucket is; its copy is reset to the start state and counts its own steps.  A bucket is
  created with as many slots as there are waiting jobs of its shape (up to `slots`) and released
  when its last job finishes.  Buckets run on their own contexts (streams), so different shapes
  overlap on the device as well.
* ``mode="per_job"``: every job its own context with the plain (unbatched) buffers of `drivers`.

Every loop iteration issues one step for every bucket (or job) before it waits on any of them;
the host decisions (a trajectory's jump choice from the FP64 norm it reads back) then wait on
that bucket's stream only.  Results do not depend on the mix: every copy of a bucket is computed
exactly as in a bucket of one, so a job's state, jump record and norms are bitwise the same alone
and in any mix (tests/test_gpu_serve.py).  Reported: per-job latency (arrival to completion)
with p50/p99, queueing delay, and aggregate site-updates/s.

Failures stay with their job.  A malformed job, or one whose footprint exceeds the whole memory
budget, is refused at admission (it would otherwise wait forever); a job whose step fails is
recorded as failed and released while the other jobs go on -- in a shared bucket a trajectory
whose norm is not finite loses its slot (reset to the start state), a library error of a
bucket's batched call fails that bucket's jobs.  Both lists come back in the stats.

The jobs are the reference examples' loops (examples/spin_model_quantum_trajectory_rk4.jl,
examples/spin_model_density_matrix.jl) as in `drivers`; the uniforms r1/r2 of a trajectory are
drawn from its own seed.
"""
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from . import batch as BT
from . import core as K
from . import drivers as DR
from . import models as Mo


@dataclass
class Job:
    kind: str            # "trajectory" (d=2, w=4) or "density" (d=4, w=8)
    na: int
    chi: int
    steps: int
    dt: float = 0.01
    seed: int = 0
    arrival: float = 0.0     # seconds after the start of the stream
    job_id: int = 0


def footprint(job, slots=1):
    """Device bytes of a job -- its MPS copies, environments and per-site scratch (complex128)
    -- or of a bucket of `slots` jobs of its shape (one context)."""
    d, w, copies = (2, 4, 7) if job.kind == "trajectory" else (4, 8, 4)
    dims = _dims(job.na, job.chi, d)
    site = sum(dims[k] * d * dims[k + 1] for k in range(job.na))
    env2 = sum(x * x for x in dims)
    scratch = 12 * max(dims[k] * d * dims[k + 1] * w for k in range(job.na))
    return 16 * (copies * site + 3 * env2 + (w + 2) * env2 + scratch) * int(slots) + (64 << 20)


def _dims(na, dmax, d):
    dims = [dmax] * (na + 1)
    dims[0] = dims[na] = 1
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
    return dims


@dataclass
class _Active:
    job: Job
    ctx: object
    buf: object
    admitted: float
    i: int = 0
    r1: np.ndarray = None
    r2: np.ndarray = None
    rec: dict = field(default_factory=dict)

    def issue(self):
        """Enqueue this job's next RK4 step (no wait)."""
        if self.job.kind == "density":
            self.buf.step()
        else:
            b = self.buf
            K.RK4stp_apply_H_half_(b.dt, b.H, b.A_coh, b.A, b.A1, b.A2, b.A3, b.env1, b.env2, b.env3, b.envop)

    def finish(self):
        """Complete the step on the host (a trajectory's norm read-back and jump decision)."""
        if self.job.kind == "trajectory":
            b, i = self.buf, self.i
            p_coh = K.normalize_lo_(b.A_coh)
            self.rec["p_coh"].append(p_coh)
            DR.trajectory_decision(b, i, p_coh, self.r1, self.r2, self.rec)
        self.i += 1
        return self.i >= self.job.steps

    def result(self):
        self.ctx.sync()
        if self.job.kind == "density":
            return {"state": self.buf.rho.sites()}
        return {"state": self.buf.A.sites(), "jumps": self.rec["jumps"], "p_coh": np.array(self.rec["p_coh"])}


def check_job(job):
    """Why a job cannot run (None when it can)."""
    if job.kind not in ("trajectory", "density"):
        return "unknown kind %r" % (job.kind,)
    if not (isinstance(job.na, int) and job.na >= 2):
        return "na must be an integer >= 2"
    if not (isinstance(job.chi, int) and job.chi >= 1):
        return "chi must be an integer >= 1"
    if not (isinstance(job.steps, int) and job.steps >= 1):
        return "steps must be an integer >= 1"
    if not (job.dt > 0 and np.isfinite(job.dt)):
        return "dt must be positive and finite"
    return None


def _start(job, ctx):
    if job.kind == "density":
        p = Mo.WaveguideChain(job.na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
        buf = DR.DensityBuffers(p, job.chi, job.dt, 8, ctx)
        return buf, None, None
    p = Mo.WaveguideChain(job.na, omega=0.5)
    buf = DR.TrajectoryBuffers(p, job.chi, job.dt, ctx)
    rng = np.random.default_rng(job.seed)
    return buf, rng.random(job.steps), rng.random(job.steps)


def _key(job):
    return (job.kind, job.na, job.chi, float(job.dt))


def _streams(job):
    rng = np.random.default_rng(job.seed)
    return rng.random(job.steps), rng.random(job.steps)


class _Bucket:
    """The bucket of one job shape (see the module docstring): batch handles on its own context,
    slots handed to jobs."""

    def __init__(self, key, nslots, device, slices, tuned=True):
        kind, na, chi, dt = key
        self.key, self.kind, self.bytes = key, kind, 0
        self.ctx = K.Context(device)
        self.eng = None
        try:
            if kind == "trajectory":
                p = Mo.WaveguideChain(na, omega=0.5)
                z = np.zeros((nslots, 1))
                self.eng = BT.TrajectoryBucket(p, chi, dt, z, z, device, ctx=self.ctx, slices=slices, tuned=tuned)
                self.eng.active[:] = False
            else:
                p = Mo.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
                self.eng = BT.DensityBucket(p, chi, dt, nslots, 8, device, ctx=self.ctx, slices=slices, tuned=tuned)
        except BaseException:
            self.close()
            raise
        self.jobs = [None] * nslots          # slot -> _Slot

    def free_slot(self):
        return next((b for b, j in enumerate(self.jobs) if j is None), None)

    def close(self):
        if self.eng is not None:
            self.eng.close()
            self.eng = None
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None


@dataclass(eq=False)
class _Slot:
    job: Job
    bucket: _Bucket
    slot: int
    admitted: float


class Server:
    """Continuous admission of jobs onto one GPU (see the module docstring).

    max_jobs: running jobs at most; hbm_bytes: device-memory budget (default 80% of what is free);
    mode: "shared" (jobs of one shape share a bucket of the batched engine) or "per_job";
    slots: copies of a shared bucket at most; slices: int8 slices of the shared buckets' larger
    contractions (0: FP64), as Context.set_precision; tuned: each shared bucket takes the
    autotuner's choice for its shape (mpsb200.autotune)."""

    def __init__(self, device=0, max_jobs=8, hbm_bytes=None, mode="shared", slots=8, slices=6, tuned=True):
        import torch
        if mode not in ("shared", "per_job"):
            raise ValueError("mode must be 'shared' or 'per_job'")
        self.device, self.max_jobs, self.mode = device, max_jobs, mode
        self.slots, self.slices, self.tuned = int(slots), int(slices), bool(tuned)
        if hbm_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_bytes = int(0.8 * free)
        self.budget = hbm_bytes

    def run(self, jobs, keep_results=False, on_admit=None):
        """Run the stream; `on_admit(handle)`, when given, is called once per admitted job after
        its buffers exist (host-side instrumentation and fault injection): the job's `_Active`
        in per_job mode, its `_Slot` (bucket and copy index) in shared mode."""
        if self.mode == "shared":
            return self._run_shared(jobs, keep_results, on_admit)
        return self._run_per_job(jobs, keep_results, on_admit)

    def _refusal(self, job):
        reason = check_job(job)
        if reason is None and footprint(job) > self.budget:
            reason = "footprint %d bytes exceeds the budget %d" % (footprint(job), self.budget)
        return reason

    @staticmethod
    def _stats(done, refused, failed, wall):
        lat = np.array([r["latency"] for r in done])
        return {"jobs": len(done), "wall_s": wall,
                "site_updates_per_s": sum(r["site_updates"] for r in done) / max(wall, 1e-9),
                "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "queue_p50_s": float(np.percentile([r["admitted"] - r["arrival"] for r in done], 50)) if done else None,
                "refused": refused, "failed": failed}

    @staticmethod
    def _record(job, admitted, t, out):
        return {"job_id": job.job_id, "kind": job.kind, "na": job.na, "chi": job.chi, "steps": job.steps,
                "arrival": job.arrival, "admitted": admitted, "finished": t, "latency": t - job.arrival,
                "site_updates": job.na * job.steps, **out}

    def _run_shared(self, jobs, keep_results, on_admit):
        pending = sorted(jobs, key=lambda j: j.arrival)
        buckets, running, done, refused, failed = [], [], [], [], []
        used = 0
        t0 = time.perf_counter()

        def drop_bucket(bk):
            nonlocal used
            buckets.remove(bk)
            used -= bk.bytes
            bk.close()

        def free(sl):
            running.remove(sl)
            sl.bucket.jobs[sl.slot] = None
            sl.bucket.eng.release(sl.slot)

        def fail_bucket(bk, e):
            for sl in [x for x in bk.jobs if x is not None]:
                failed.append({"job_id": sl.job.job_id, "step": int(bk.eng.t[sl.slot]), "error": str(e)})
                running.remove(sl)
            drop_bucket(bk)

        while pending or running:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now and len(running) < self.max_jobs:
                job = pending[0]
                reason = self._refusal(job)
                if reason is not None:
                    pending.pop(0)
                    refused.append({"job_id": job.job_id, "reason": reason})
                    continue
                key = _key(job)
                bk = next((b for b in buckets if b.key == key and b.free_slot() is not None), None)
                if bk is None:
                    waiting = sum(1 for j in pending if j.arrival <= now and _key(j) == key)
                    n = max(1, min(self.slots, waiting, self.max_jobs - len(running)))
                    while n > 1 and used + footprint(job, n) > self.budget:
                        n -= 1
                    if used + footprint(job, n) > self.budget:
                        break
                    try:
                        bk = _Bucket(key, n, self.device, self.slices, self.tuned)
                    except _lib.MpsbError as e:
                        pending.pop(0)
                        failed.append({"job_id": job.job_id, "step": -1, "error": str(e)})
                        continue
                    bk.bytes = footprint(job, n)
                    used += bk.bytes
                    buckets.append(bk)
                pending.pop(0)
                b = bk.free_slot()
                sl = _Slot(job, bk, b, time.perf_counter() - t0)
                try:
                    if job.kind == "trajectory":
                        bk.eng.assign(b, *_streams(job))
                    else:
                        bk.eng.assign(b)
                    bk.jobs[b] = sl
                    running.append(sl)
                    if on_admit is not None:
                        on_admit(sl)
                except _lib.MpsbError as e:
                    failed.append({"job_id": job.job_id, "step": -1, "error": str(e)})
                    if sl in running:
                        free(sl)
                    else:
                        bk.eng.release(b)
                    if not any(bk.jobs):
                        drop_bucket(bk)
            if not running:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - now)))
                continue
            live = [bk for bk in buckets if any(bk.jobs)]
            for bk in live:
                try:
                    bk.eng.issue()
                except _lib.MpsbError as e:
                    fail_bucket(bk, e)
            for bk in [x for x in live if x in buckets]:
                bad = []
                try:
                    bk.eng.finish(bad)
                except _lib.MpsbError as e:
                    fail_bucket(bk, e)
                    continue
                for b in bad:
                    sl = bk.jobs[b]
                    failed.append({"job_id": sl.job.job_id, "step": int(bk.eng.t[b]),
                                   "error": "MPSB_ERR_NONFINITE: the trajectory's norm is not finite"})
                    free(sl)
                    bk.eng.reset(b)
                for b, sl in enumerate(bk.jobs):
                    if sl is None or bk.eng.t[b] < sl.job.steps:
                        continue
                    out = {}
                    if keep_results:
                        out["state"] = bk.eng.state(b)
                        if sl.job.kind == "trajectory":
                            out["jumps"] = list(bk.eng.jumps[b])
                            out["p_coh"] = np.array(bk.eng.p_coh[b])
                    done.append(self._record(sl.job, sl.admitted, time.perf_counter() - t0, out))
                    free(sl)
                if not any(bk.jobs):
                    drop_bucket(bk)
        for bk in list(buckets):
            drop_bucket(bk)
        return done, self._stats(done, refused, failed, time.perf_counter() - t0)

    def _run_per_job(self, jobs, keep_results, on_admit):
        pending = sorted(jobs, key=lambda j: j.arrival)
        active, done, refused, failed, used = [], [], [], [], 0
        t0 = time.perf_counter()

        def release(a):
            nonlocal used
            active.remove(a)
            used -= footprint(a.job)
            a.buf = None          # the job's device buffers go before its context
            a.ctx.close()

        while pending or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now and len(active) < self.max_jobs:
                reason = self._refusal(pending[0])
                if reason is not None:
                    job = pending.pop(0)
                    refused.append({"job_id": job.job_id, "reason": reason})
                    continue
                if used + footprint(pending[0]) > self.budget:
                    break
                job = pending.pop(0)
                ctx = a = None
                try:   # a failure while setting the job up stays with the job
                    ctx = K.Context(self.device)
                    buf, r1, r2 = _start(job, ctx)
                    a = _Active(job, ctx, buf, time.perf_counter() - t0, r1=r1, r2=r2,
                                rec={"p_coh": [], "jumps": []})
                    active.append(a)
                    used += footprint(job)
                    if on_admit is not None:
                        on_admit(a)
                except _lib.MpsbError as e:
                    failed.append({"job_id": job.job_id, "step": -1, "error": str(e)})
                    if a is not None and a in active:
                        release(a)
                    elif ctx is not None:
                        ctx.close()
            if not active:
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - now)))
                continue
            for a in list(active):
                try:
                    a.issue()
                except _lib.MpsbError as e:
                    failed.append({"job_id": a.job.job_id, "step": a.i, "error": str(e)})
                    release(a)
            finished = []
            for a in list(active):
                try:
                    if a.finish():
                        finished.append(a)
                except _lib.MpsbError as e:
                    failed.append({"job_id": a.job.job_id, "step": a.i, "error": str(e)})
                    release(a)
            for a in finished:
                out = a.result() if keep_results else {}
                done.append(self._record(a.job, a.admitted, time.perf_counter() - t0, out))
                release(a)
        return done, self._stats(done, refused, failed, time.perf_counter() - t0)


def poisson_jobs(n, rate, seed, kinds=(0.7, 0.3), traj_na=(20, 40), traj_chi=(16, 32, 64),
                 rho_na=(8, 16), rho_chi=(16, 32), steps=(10, 30), dt=0.01):
    """A seeded mixed stream: exponential inter-arrival times at `rate` jobs/s, a fraction
    kinds[0] of trajectories, sizes drawn uniformly from the given ranges / sets."""
    rng = np.random.default_rng(seed)
    t, jobs = 0.0, []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if rng.random() < kinds[0]:
            jobs.append(Job("trajectory", int(rng.integers(traj_na[0], traj_na[1] + 1)), int(rng.choice(traj_chi)),
                            int(rng.integers(steps[0], steps[1] + 1)), dt, seed * 100003 + i, t, i))
        else:
            jobs.append(Job("density", int(rng.integers(rho_na[0], rho_na[1] + 1)), int(rng.choice(rho_chi)),
                            int(rng.integers(steps[0], steps[1] + 1)), dt / 2, seed * 100003 + i, t, i))
    return jobs
