"""Host logic of the continuous-batching serving loop (shared buckets), on CPU: the batched
engine behind a bucket is replaced by a fake that counts steps, so admission, slot reuse, bucket
lifetime and per-job failure handling are checked without a device."""
import numpy as np
import pytest


class FakeEngine:
    """Stands in for batch.TrajectoryBucket / DensityBucket: per-copy step counters; a copy whose
    job was marked bad reports a non-finite norm at its next step."""

    def __init__(self, nslots, log):
        self.t = np.zeros(nslots, dtype=np.int64)
        self.active = np.zeros(nslots, dtype=bool)
        self.bad_next = set()
        self.jumps = [[] for _ in range(nslots)]
        self.p_coh = [[] for _ in range(nslots)]
        self.log = log

    def assign(self, b, *streams):
        self.t[b] = 0
        self.active[b] = True
        self.jumps[b], self.p_coh[b] = [], []
        self.log.append(("assign", b))

    def release(self, b):
        self.active[b] = False

    def reset(self, b):
        self.log.append(("reset", b))

    def issue(self):
        pass

    def finish(self, bad=None):
        import time
        time.sleep(0.002)
        for b in range(len(self.t)):
            if not self.active[b]:
                continue
            if b in self.bad_next and bad is not None:
                self.bad_next.discard(b)
                bad.append(b)
                self.active[b] = False
                continue
            self.p_coh[b].append(1.0)
            self.t[b] += 1

    def state(self, b):
        return [np.full((1, 2, 1), float(b))]

    def close(self):
        self.log.append(("close",))


@pytest.fixture
def fake_buckets(monkeypatch):
    from mpsb200 import serve as S
    made = []

    class FakeBucket:
        def __init__(self, key, nslots, device, slices, tuned=True):
            self.key, self.kind, self.bytes = key, key[0], 0
            self.log = []
            self.eng = FakeEngine(nslots, self.log)
            self.jobs = [None] * nslots
            self.nslots = nslots
            self.closed = False
            made.append(self)

        def free_slot(self):
            return next((b for b, j in enumerate(self.jobs) if j is None), None)

        def close(self):
            self.closed = True

    monkeypatch.setattr(S, "_Bucket", FakeBucket)
    return made


def test_jobs_of_one_shape_share_a_bucket_sized_by_the_waiting_jobs(fake_buckets):
    from mpsb200 import serve as S
    jobs = [S.Job("trajectory", 10, 16, 3 + i, 0.01, i, 0.0, i) for i in range(3)]
    jobs.append(S.Job("density", 6, 8, 2, 0.005, 9, 0.0, 3))
    done, stats = S.Server(max_jobs=8, slots=4, hbm_bytes=1 << 40).run(jobs, keep_results=True)
    assert stats["failed"] == [] and stats["refused"] == [] and stats["jobs"] == 4
    traj = [b for b in fake_buckets if b.kind == "trajectory"]
    assert len(traj) == 1 and traj[0].nslots == 3          # one bucket, as many copies as waiting jobs
    assert all(b.closed for b in fake_buckets)             # released with their last job
    for r in done:
        assert r["steps"] == next(j.steps for j in jobs if j.job_id == r["job_id"])
        if r["kind"] == "trajectory":
            assert len(r["p_coh"]) == r["steps"]


def test_a_later_job_takes_the_copy_a_finished_job_left(fake_buckets):
    from mpsb200 import serve as S
    seen = {}

    def admit(sl):
        seen[sl.job.job_id] = (id(sl.bucket), sl.slot)

    jobs = [S.Job("trajectory", 10, 16, 2, 0.01, 0, 0.0, 0),     # leaves after two steps
            S.Job("trajectory", 10, 16, 60, 0.01, 1, 0.0, 1),    # keeps the bucket running
            S.Job("trajectory", 10, 16, 3, 0.01, 2, 0.05, 2)]    # arrives later
    done, stats = S.Server(max_jobs=8, slots=4, hbm_bytes=1 << 40).run(jobs, on_admit=admit)
    assert stats["jobs"] == 3 and len(fake_buckets) == 1
    assert seen[2] == seen[0]                                   # same bucket, the freed copy
    assert fake_buckets[0].log.count(("assign", seen[0][1])) == 2


def test_a_non_finite_copy_fails_its_job_alone(fake_buckets):
    from mpsb200 import serve as S

    def admit(sl):
        if sl.job.job_id == 1:
            sl.bucket.eng.bad_next.add(sl.slot)

    jobs = [S.Job("trajectory", 10, 16, 4, 0.01, i, 0.0, i) for i in range(3)]
    done, stats = S.Server(max_jobs=8, slots=4, hbm_bytes=1 << 40).run(jobs, on_admit=admit)
    assert [(f["job_id"], f["step"]) for f in stats["failed"]] == [(1, 0)]
    assert sorted(r["job_id"] for r in done) == [0, 2]
    assert ("reset", 1) in fake_buckets[0].log                  # the failed copy back at the start state


def test_a_bucket_waits_for_memory_and_the_queue_keeps_order(fake_buckets):
    from mpsb200 import serve as S
    a = S.Job("trajectory", 40, 64, 5, 0.01, 0, 0.0, 0)
    b = S.Job("density", 30, 64, 2, 0.005, 1, 0.0, 1)
    budget = max(S.footprint(a), S.footprint(b)) + 1            # one bucket at a time
    order = []
    done, stats = S.Server(max_jobs=8, slots=4, hbm_bytes=budget).run(
        [a, b], on_admit=lambda sl: order.append(sl.job.job_id))
    assert stats["jobs"] == 2 and order == [0, 1]
    assert done[0]["job_id"] == 0 and done[1]["admitted"] >= done[0]["finished"] - 1e-3
