"""The batched engine's per-bucket autotuner: table lookup and how a bucket applies it (host
logic, no device), and on the GPU that a tuned bucket keeps every copy batch-independent."""
import numpy as np
import pytest

TABLE = {"entries": [
    {"kind": "trajectory", "na": 64, "d": 2, "w": 4, "chi": 16, "slices": 0, "min_flops": 0.0},
    {"kind": "trajectory", "na": 64, "d": 2, "w": 4, "chi": 64, "slices": 6, "min_flops": 2.0 ** 25},
    {"kind": "trajectory", "na": 64, "d": 2, "w": 4, "chi": 256, "slices": 6, "min_flops": 2.0 ** 22},
    {"kind": "density", "na": 40, "d": 4, "w": 8, "chi": 128, "slices": 6, "min_flops": 2.0 ** 23},
]}


class FakeCtx:
    def __init__(self):
        self.calls = []

    def set_precision(self, s, min_tiles=64):
        self.calls.append(("precision", s))

    def set_batched_split_threshold(self, th):
        self.calls.append(("threshold", th))


def test_lookup_takes_the_nearest_cap_of_the_same_shape_family():
    from mpsb200 import autotune as AT
    assert AT.lookup("trajectory", 2, 4, 256, TABLE) == (6, 2.0 ** 22)
    assert AT.lookup("trajectory", 2, 4, 200, TABLE) == (6, 2.0 ** 22)    # log-nearest: 256
    assert AT.lookup("trajectory", 2, 4, 100, TABLE) == (6, 2.0 ** 25)    # 64
    assert AT.lookup("trajectory", 2, 4, 32, TABLE) == (0, 0.0)           # tie 16 / 64 -> smaller cap
    assert AT.lookup("density", 4, 8, 300, TABLE) == (6, 2.0 ** 23)
    assert AT.lookup("density", 4, 6, 128, TABLE) is None                 # other MPO width
    assert AT.lookup("trajectory", 2, 4, 64, {"entries": []}) is None


def test_apply_sets_the_tuned_precision_and_threshold():
    from mpsb200 import autotune as AT
    c = FakeCtx()
    assert AT.apply(c, "trajectory", 2, 4, 250, 6, TABLE) == 6
    assert c.calls == [("precision", 6), ("threshold", 2.0 ** 22)]
    c = FakeCtx()
    assert AT.apply(c, "trajectory", 2, 4, 16, 6, TABLE) == 0             # the tuner chose FP64
    assert c.calls == [("precision", 0)]
    c = FakeCtx()
    assert AT.apply(c, "trajectory", 2, 4, 64, 0, TABLE) == 0             # FP64 asked: no lookup
    assert c.calls == [("precision", 0)]
    c = FakeCtx()
    assert AT.apply(c, "density", 4, 6, 64, 6, TABLE) == 6                # no entry: as asked
    assert c.calls == [("precision", 6)]


def test_committed_table_covers_the_benchmarked_shapes():
    from mpsb200 import autotune as AT
    table = AT.load_table()
    if table is None:
        pytest.skip("no tuning table committed")
    caps = {e["chi"] for e in table["entries"] if e["kind"] == "trajectory"}
    assert set(AT.TRAJ_CAPS) <= caps
    for e in table["entries"]:
        assert e["slices"] in (0, 3, 4, 5, 6, 7) and e["min_flops"] >= 0
        best = min(e["ms_per_step"].values())
        assert e["ms_per_step"]["%d:%g" % (e["slices"], e["min_flops"])] == best


@pytest.mark.gpu
def test_tuned_buckets_compute_each_trajectory_the_same_alone_and_shared(gpu_ctx):
    from mpsb200 import batch as BT
    from mpsb200 import models as GM
    p = GM.WaveguideChain(12, omega=0.5)
    rng = np.random.default_rng(8)
    n, caps = 6, [16, 16, 16, 48, 48]
    r1, r2 = rng.random((len(caps), n)) * 0.97, rng.random((len(caps), n))
    shared = BT.TrajectoryBatch(p, caps, 0.01, r1, r2, slices=6, tuned=True)
    for _ in range(n):
        shared.step()
    for k in (0, 3):
        alone = BT.TrajectoryBatch(p, [caps[k]], 0.01, r1[k:k + 1], r2[k:k + 1], slices=6, tuned=True)
        for _ in range(n):
            alone.step()
        a, b = shared.records(k), alone.records(0)
        assert np.array_equal(a[0], b[0]) and a[1] == b[1]
        assert all(np.array_equal(x, y) for x, y in zip(a[2], b[2]))
        alone.close()
    shared.close()
