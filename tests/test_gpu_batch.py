"""Batched trajectories (mpsb200.batch): many trajectories per bond-dim bucket, every kernel over
all copies of a bucket at once.

* a trajectory's p_coh record, jump record and final state are bitwise the same in a bucket of
  one and in a bucket shared with others (and with other buckets running beside it);
* against the oracle's example loop (oracle/drivers.run_trajectory) with the same uniforms:
  identical jump records (forced jump steps exercise both waveguide jumps) and p_coh within
  1e-10 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _uniforms(seed, nsteps, forced=()):
    g = np.random.default_rng(seed)
    r1, r2 = g.random(nsteps), g.random(nsteps)
    for i in forced:
        r1[i] = 1.0 - 1e-12   # above any p_coh < 1: a jump step
    return r1, r2


def _run(p, chis, dt, nsteps, seeds, forced, slices=0):
    from mpsb200 import batch as BT
    r = [_uniforms(s, nsteps, forced) for s in seeds]
    tb = BT.TrajectoryBatch(p, chis, dt, [x[0] for x in r], [x[1] for x in r], slices=slices)
    try:
        for _ in range(nsteps):
            tb.step()
        return [tb.records(k) for k in range(len(chis))], r
    finally:
        tb.close()


def test_batched_equals_alone_bitwise():
    from mpsb200 import models as GM
    p = GM.WaveguideChain(10, omega=0.5)
    chis, seeds, forced = [8, 16, 8, 16, 8], [0, 1, 2, 3, 4], (3, 7)
    mixed, _ = _run(p, chis, 0.01, 12, seeds, forced)
    for k, (c, s) in enumerate(zip(chis, seeds)):
        alone, _ = _run(p, [c], 0.01, 12, [s], forced)
        pc, jm, st = mixed[k]
        pa, ja, sa = alone[0]
        assert np.array_equal(pc, pa) and jm == ja
        assert all(np.array_equal(x, y) for x, y in zip(st, sa))


def test_batched_matches_oracle_jump_records():
    from mpsb200 import models as GM
    from oracle import drivers as ODR
    from oracle import models as OM
    na, dt, n = 10, 0.01, 12
    chis, seeds, forced = [8, 8, 16], [5, 6, 7], (2, 5, 9)
    from gpu_util import perturbed_oracle_qr
    got, unif = _run(GM.WaveguideChain(na, omega=0.5), chis, dt, n, seeds, forced)
    for k, c in enumerate(chis):
        r1, r2 = unif[k]
        rec = ODR.run_trajectory(OM.SpinChain(na, omega=0.5), c, dt, n, r1, r2, measure_int=n)
        with perturbed_oracle_qr(1e-15):
            pert = ODR.run_trajectory(OM.SpinChain(na, omega=0.5), c, dt, n, r1, r2, measure_int=n)
        env = np.abs(pert["p_coh"] - rec["p_coh"])
        pc, jm, _ = got[k]
        assert [(j[0], j[1], j[2]) for j in jm] == [(j[0], j[1], j[2]) for j in rec["jumps"]]
        assert len(jm) == len(forced)
        # the oracle's own spread under rounding-level perturbations bounds any implementation
        assert np.all(np.abs(pc - rec["p_coh"]) <= 100 * env + 1e-12)


def test_batched_split_precision_equals_alone_and_stays_near_fp64():
    """The sliced tensor-core path inside batched buckets (N=14, bonds up to 128): bitwise the
    same alone and in a shared bucket, and within 1e-9 of the FP64 batched run on p_coh."""
    from mpsb200 import models as GM
    p = GM.WaveguideChain(14, omega=0.5)
    chis, seeds, forced = [128, 64, 128], [8, 9, 10], (4,)
    mixed, _ = _run(p, chis, 0.01, 8, seeds, forced, slices=6)
    fp, _ = _run(p, chis, 0.01, 8, seeds, forced, slices=0)
    for k, (c, s) in enumerate(zip(chis, seeds)):
        alone, _ = _run(p, [c], 0.01, 8, [s], forced, slices=6)
        assert np.array_equal(mixed[k][0], alone[0][0]) and mixed[k][1] == alone[0][1]
        assert all(np.array_equal(x, y) for x, y in zip(mixed[k][2], alone[0][2]))
        assert [j[:3] for j in mixed[k][1]] == [j[:3] for j in fp[k][1]]
        assert np.abs(mixed[k][0] - fp[k][0]).max() <= 1e-9
        assert any(np.abs(x - y).max() > 0 for x, y in zip(mixed[k][2], fp[k][2]))   # the path is taken
