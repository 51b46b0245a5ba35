"""Serving loop: a stream of trajectory and density-matrix jobs sharing one GPU.

Jobs arrive over time (seeded Poisson arrivals); a job is admitted as soon as a slot is free
and its device footprint fits in the memory budget, gets its own context (its own CUDA
streams and scratch), and keeps its MPS state on the device until it finishes.  Every loop
iteration issues one RK4 step for every active job before it waits on any of them, so the
jobs' kernels overlap on the device; the per-job host decisions (a trajectory's jump choice
from the FP64 norm it reads back) then wait on that job's stream only.  Results do not depend
on the mix: every job's arithmetic is its own (tests/test_gpu_serve.py checks bitwise
equality alone vs in the mix).  Reported: per-job latency (arrival to completion) with
p50/p99, queueing delay, and aggregate site-updates/s.

Failures stay with their job.  A malformed job, or one whose footprint exceeds the whole
memory budget, is refused at admission (it would otherwise wait forever); a job whose step
fails (a library error, e.g. a NaN norm) is recorded as failed, its buffers and context are
released, and the other jobs go on.  Both lists come back in the stats.

The jobs are the reference examples' loops (examples/spin_model_quantum_trajectory_rk4.jl,
examples/spin_model_density_matrix.jl) as in `drivers`; the uniforms r1/r2 of a trajectory are
drawn from its own seed.
"""
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
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


def footprint(job):
    """Device bytes of a job: its MPS copies, environments and per-site scratch (complex128)."""
    d, w, copies = (2, 4, 7) if job.kind == "trajectory" else (4, 8, 4)
    dims = _dims(job.na, job.chi, d)
    site = sum(dims[k] * d * dims[k + 1] for k in range(job.na))
    env2 = sum(x * x for x in dims)
    scratch = 12 * max(dims[k] * d * dims[k + 1] * w for k in range(job.na))
    return 16 * (copies * site + 3 * env2 + (w + 2) * env2 + scratch) + (64 << 20)


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


class Server:
    """Continuous admission of jobs onto one GPU (see the module docstring)."""

    def __init__(self, device=0, max_jobs=8, hbm_bytes=None):
        import torch
        self.device, self.max_jobs = device, max_jobs
        if hbm_bytes is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_bytes = int(0.8 * free)
        self.budget = hbm_bytes

    def run(self, jobs, keep_results=False, on_admit=None):
        """Run the stream; `on_admit(active_job)`, when given, is called once per admitted job
        after its buffers exist (host-side instrumentation and fault injection)."""
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
                reason = check_job(pending[0])
                if reason is None and footprint(pending[0]) > self.budget:
                    reason = "footprint %d bytes exceeds the budget %d" % (footprint(pending[0]), self.budget)
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
                t = time.perf_counter() - t0
                done.append({"job_id": a.job.job_id, "kind": a.job.kind, "na": a.job.na, "chi": a.job.chi,
                             "steps": a.job.steps, "arrival": a.job.arrival, "admitted": a.admitted,
                             "finished": t, "latency": t - a.job.arrival, "site_updates": a.job.na * a.job.steps,
                             **out})
                release(a)
        wall = time.perf_counter() - t0
        lat = np.array([r["latency"] for r in done])
        stats = {"jobs": len(done), "wall_s": wall,
                 "site_updates_per_s": sum(r["site_updates"] for r in done) / max(wall, 1e-9),
                 "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                 "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                 "queue_p50_s": float(np.percentile([r["admitted"] - r["arrival"] for r in done], 50)) if done else None,
                 "refused": refused, "failed": failed}
        return done, stats


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
