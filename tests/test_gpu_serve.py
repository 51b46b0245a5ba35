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


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_the_mix(gpu_ctx):
    from mpsb200 import serve as S
    jobs = S.poisson_jobs(6, 200.0, 3, traj_na=(10, 14), traj_chi=(8, 16), rho_na=(6, 8), rho_chi=(8, 16),
                          steps=(6, 12))
    mix, stats = S.Server(max_jobs=4).run(jobs, keep_results=True)
    assert stats["jobs"] == len(jobs)
    assert stats["latency_p99_s"] >= stats["latency_p50_s"] > 0
    for r in mix:
        job = next(j for j in jobs if j.job_id == r["job_id"])
        alone, _ = S.Server(max_jobs=1).run([dataclasses.replace(job, arrival=0.0)], keep_results=True)
        a = alone[0]
        assert all(np.array_equal(x, y) for x, y in zip(r["state"], a["state"]))
        if r["kind"] == "trajectory":
            assert r["jumps"] == a["jumps"] and np.array_equal(r["p_coh"], a["p_coh"])
