"""Serving loop (the mixed-stream configuration): continuous admission, overlap on one GPU,
and results that are the same alone and in the mix."""
import dataclasses

import numpy as np
import pytest


def test_stream_is_seeded_and_mixed():
    from mpsb200 import serve as S
    a = S.poisson_jobs(40, 200.0, 7)
    b = S.poisson_jobs(40, 200.0, 7)
    assert a == b
    kinds = [j.kind for j in a]
    assert 0 < kinds.count("density") < len(a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    assert all(S.footprint(j) > 0 for j in a)


def test_malformed_and_oversize_jobs_are_refused_at_admission():
    """Host-side failure handling (no device needed: refused jobs never get a context): a
    malformed descriptor and a job larger than the whole budget are refused with a reason,
    instead of blocking the stream forever."""
    from mpsb200 import serve as S
    jobs = [S.Job("trajectory", 20, 32, 10, job_id=0), S.Job("rk5", 20, 32, 10, job_id=1),
            S.Job("density", 1, 16, 10, job_id=2), S.Job("trajectory", 20, 32, 0, job_id=3),
            S.Job("density", 8, 16, 10, dt=float("nan"), job_id=4)]
    budget = S.footprint(jobs[0]) - 1            # smaller than the one well-formed job
    done, stats = S.Server(max_jobs=2, hbm_bytes=budget).run(jobs)
    assert done == [] and stats["failed"] == []
    reasons = {r["job_id"]: r["reason"] for r in stats["refused"]}
    assert sorted(reasons) == [0, 1, 2, 3, 4]
    assert "exceeds the budget" in reasons[0] and "kind" in reasons[1] and "na" in reasons[2]
    assert "steps" in reasons[3] and "dt" in reasons[4]


def test_a_job_whose_setup_fails_is_recorded_and_the_stream_goes_on(monkeypatch):
    """A library error while a job's context or buffers are created (here: a fake context whose
    creation fails, so no device is needed) fails that job at step -1; the loop returns."""
    from mpsb200 import _lib
    from mpsb200 import serve as S

    class FailingContext:
        def __init__(self, device=0):
            raise _lib.MpsbError(-4, "mpsb_ctx_create", "out of memory (injected)")

    monkeypatch.setattr(S.K, "Context", FailingContext)
    jobs = [S.Job("trajectory", 20, 16, 3, job_id=0), S.Job("density", 8, 16, 3, job_id=1)]
    done, stats = S.Server(max_jobs=2, hbm_bytes=1 << 40).run(jobs)
    assert done == [] and stats["refused"] == []
    assert [(f["job_id"], f["step"]) for f in stats["failed"]] == [(0, -1), (1, -1)]
    assert all("injected" in f["error"] for f in stats["failed"])


@pytest.mark.gpu
def test_a_failing_job_leaves_the_others_intact(gpu_ctx):
    """Fault injected from the host: one trajectory's Hamiltonian gets a NaN after admission.
    Its norm check fails (MPSB_ERR_NONFINITE), it is recorded as failed and released, and the
    other jobs finish with the results they have without it."""
    from mpsb200 import serve as S
    jobs = S.poisson_jobs(5, 200.0, 5, kinds=(1.0, 0.0), traj_na=(10, 12), traj_chi=(8, 16), steps=(6, 10))
    bad = jobs[2].job_id

    def corrupt(a):
        if a.job.job_id == bad:
            a.buf.H[0].set_site(0, a.buf.H[0].site(0) * np.nan)

    mixed, stats = S.Server(max_jobs=3, mode="per_job").run(jobs, keep_results=True, on_admit=corrupt)
    assert [f["job_id"] for f in stats["failed"]] == [bad] and "NONFINITE" in stats["failed"][0]["error"]
    clean, _ = S.Server(max_jobs=3, mode="per_job").run([j for j in jobs if j.job_id != bad], keep_results=True)
    assert sorted(r["job_id"] for r in mixed) == sorted(r["job_id"] for r in clean)
    for r in mixed:
        c = next(x for x in clean if x["job_id"] == r["job_id"])
        assert all(np.array_equal(x, y) for x, y in zip(r["state"], c["state"]))


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_the_mix(gpu_ctx):
    from mpsb200 import serve as S
    jobs = S.poisson_jobs(6, 200.0, 3, traj_na=(10, 14), traj_chi=(8, 16), rho_na=(6, 8), rho_chi=(8, 16),
                          steps=(6, 12))
    mix, stats = S.Server(max_jobs=4, mode="per_job").run(jobs, keep_results=True)
    assert stats["jobs"] == len(jobs)
    assert stats["latency_p99_s"] >= stats["latency_p50_s"] > 0
    for r in mix:
        job = next(j for j in jobs if j.job_id == r["job_id"])
        alone, _ = S.Server(max_jobs=1, mode="per_job").run([dataclasses.replace(job, arrival=0.0)],
                                                             keep_results=True)
        a = alone[0]
        assert all(np.array_equal(x, y) for x, y in zip(r["state"], a["state"]))
        if r["kind"] == "trajectory":
            assert r["jumps"] == a["jumps"] and np.array_equal(r["p_coh"], a["p_coh"])


def _shape_mix(n, seed):
    """A stream whose jobs repeat a few shapes, so shared buckets hold several jobs at once and
    jobs join a bucket that is already running (later arrivals, other step counts)."""
    from mpsb200 import serve as S
    rng = np.random.default_rng(seed)
    shapes = [("trajectory", 10, 16, 0.01), ("trajectory", 12, 8, 0.01), ("density", 6, 16, 0.005)]
    jobs, t = [], 0.0
    for i in range(n):
        kind, na, chi, dt = shapes[int(rng.integers(len(shapes)))]
        t += rng.exponential(1.0 / 400.0)
        jobs.append(S.Job(kind, na, chi, int(rng.integers(5, 12)), dt, 1000 + i, t, i))
    return jobs


@pytest.mark.gpu
def test_shared_buckets_results_are_the_same_alone_and_in_the_mix(gpu_ctx):
    """Continuous batching: jobs of one shape share the batched engine's bucket, join it while it
    runs, and leave it at their own step count; every job's state, jump record and norms are
    bitwise those of the job run alone."""
    from mpsb200 import serve as S
    jobs = _shape_mix(12, 21)
    shared = {}

    def seen(sl):
        shared.setdefault(id(sl.bucket), set()).add(sl.job.job_id)

    mix, stats = S.Server(max_jobs=8, slots=4).run(jobs, keep_results=True, on_admit=seen)
    assert stats["jobs"] == len(jobs) and stats["failed"] == [] and stats["refused"] == []
    assert max(len(v) for v in shared.values()) >= 3       # some bucket carried several jobs
    for r in mix:
        job = next(j for j in jobs if j.job_id == r["job_id"])
        alone, _ = S.Server(max_jobs=1, slots=4).run([dataclasses.replace(job, arrival=0.0)], keep_results=True)
        a = alone[0]
        assert all(np.array_equal(x, y) for x, y in zip(r["state"], a["state"]))
        if r["kind"] == "trajectory":
            assert r["jumps"] == a["jumps"] and np.array_equal(r["p_coh"], a["p_coh"])


@pytest.mark.gpu
def test_shared_bucket_failing_trajectory_leaves_its_bucket_mates_intact(gpu_ctx):
    """Fault injected from the host: one trajectory's copy in a shared bucket gets a NaN site
    after admission.  Its norm is not finite, so that job fails and its slot is reset; the jobs
    sharing the bucket finish with the results they have without it."""
    from mpsb200 import serve as S
    jobs = [S.Job("trajectory", 10, 16, 8, 0.01, 500 + i, 0.0, i) for i in range(4)]
    bad = 2

    def corrupt(sl):
        if sl.job.job_id == bad:
            site = sl.bucket.eng.A.site_copy(sl.slot, 3)
            sl.bucket.eng.A.set_site_copy(sl.slot, 3, site * np.nan)

    mixed, stats = S.Server(max_jobs=4, slots=4).run(jobs, keep_results=True, on_admit=corrupt)
    assert [(f["job_id"], f["step"]) for f in stats["failed"]] == [(bad, 0)]
    assert "NONFINITE" in stats["failed"][0]["error"]
    clean, _ = S.Server(max_jobs=4, slots=4).run([j for j in jobs if j.job_id != bad], keep_results=True)
    assert sorted(r["job_id"] for r in mixed) == sorted(r["job_id"] for r in clean) == [0, 1, 3]
    for r in mixed:
        c = next(x for x in clean if x["job_id"] == r["job_id"])
        assert all(np.array_equal(x, y) for x, y in zip(r["state"], c["state"]))
        assert np.array_equal(r["p_coh"], c["p_coh"]) and r["jumps"] == c["jumps"]
