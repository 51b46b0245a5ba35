"""Per-bucket autotuner of the batched engine.

A bucket (`batch.TrajectoryBucket`, `batch.DensityBucket`) runs every contraction of its copies
as one batched call, and each GEMM of a batched call picks its kernel from one copy's problem
alone: the int8-sliced tensor-core path (`slices` > 0) when 8 M N K >= `min_flops`, the FP64
DMMA path otherwise.  Which threshold is fastest depends on the bucket's shape (bond cap chi,
local dimension d, MPO width w): the sliced path pays four slicing launches per GEMM, which small
problems do not earn back.  The tuner times whole steps of a bucket for each candidate
(slices, min_flops) on the device it runs on and records the fastest; the table it writes
(`tuning_b200.json`, measured on one B200) is looked up by shape when a bucket is created.

The choice depends only on the bucket's shape, never on its number of copies, so a trajectory
computes the same bits in a bucket of any size (the engine's batch-independence is kept).

    python -m mpsb200.autotune [--out PATH] [--copies B] [--steps K]
"""
import json
import math
import os
import time

TABLE_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json")

# (slices, min_flops): the sliced path from that many flops of one copy's GEMM, or FP64 only
CANDIDATES = ((6, 2.0 ** 22), (6, 2.0 ** 23), (6, 2.0 ** 24), (6, 2.0 ** 25), (6, 2.0 ** 26), (0, 0.0))

# the shapes tuned by default: the batching workload's trajectory caps (N=64, d=2, w=4) and the
# serving stream's density-matrix caps (d=4, w=8)
TRAJ_CAPS = [int(round(8 * 32 ** (j / 15.0))) for j in range(16)]
RHO_CAPS = [32, 64, 128, 256]

_cache = {}


def load_table(path=None):
    """The tuning table (a dict with an "entries" list), or None when the file is absent."""
    path = path or TABLE_PATH
    if path not in _cache:
        if not os.path.exists(path):
            return None
        with open(path) as f:
            _cache[path] = json.load(f)
    return _cache[path]


def lookup(kind, d, w, chi, table=None):
    """(slices, min_flops) of the table entry of this kind, d and w whose cap is nearest to chi
    (in log scale; the smaller cap on a tie), or None without a table or entry."""
    table = table if table is not None else load_table()
    if not table:
        return None
    best = None
    for e in table.get("entries", []):
        if e["kind"] != kind or int(e["d"]) != int(d) or int(e["w"]) != int(w):
            continue
        dist = round(abs(math.log2(float(e["chi"])) - math.log2(float(chi))), 9)
        key = (dist, int(e["chi"]))
        if best is None or key < best[0]:
            best = (key, (int(e["slices"]), float(e["min_flops"])))
    return None if best is None else best[1]


def apply(ctx, kind, d, w, chi, slices, table=None):
    """Set ctx's precision for a bucket of this shape: with slices > 0 the tuned (slices,
    min_flops) of the shape when the table (default: the committed one) has it, else `slices`
    with the default threshold; slices = 0 stays FP64.  Returns the slices in effect."""
    hit = lookup(kind, d, w, chi, table) if slices else None
    if hit is None:
        ctx.set_precision(slices)
        return slices
    s, th = hit
    ctx.set_precision(s)
    if s:
        ctx.set_batched_split_threshold(th)
    return s


def _time_bucket(bk, steps, warmup):
    import torch
    for _ in range(warmup):
        bk.issue()
        bk.finish()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        bk.issue()
        bk.finish()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1e3 / steps


def tune(kind, na, chi, copies, steps=2, warmup=2, device=0, candidates=CANDIDATES):
    """Milliseconds per step of one bucket for every candidate; the fastest is the choice."""
    import numpy as np

    from . import batch as BT
    from . import core as K
    from . import models as Mo
    ctx = K.Context(device)
    try:
        if kind == "trajectory":
            p = Mo.WaveguideChain(na, omega=0.5)
            n = (warmup + steps) * len(candidates) + 1
            rng = np.random.default_rng(chi)
            # r1 = 0 < p_coh: no copy jumps, every step is the coherent RK4 step
            bk = BT.TrajectoryBucket(p, chi, 0.01, np.zeros((copies, n)), rng.random((copies, n)), device, ctx=ctx)
            d, w = 2, 4
        else:
            p = Mo.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
            bk = BT.DensityBucket(p, chi, 0.005, copies, 8, device, ctx=ctx)
            for b in range(copies):
                bk.assign(b)
            d, w = 4, 8
        ms = {}
        for s, th in candidates:
            ctx.set_precision(s)
            ctx.set_batched_split_threshold(th if s else 2.0 ** 24)
            ms["%d:%g" % (s, th)] = _time_bucket(bk, steps, warmup)
        bk.close()
    finally:
        ctx.close()
    (s, th), best = min(((c, ms["%d:%g" % c]) for c in candidates), key=lambda x: x[1])
    return {"kind": kind, "na": na, "d": d, "w": w, "chi": chi, "copies": copies, "slices": s,
            "min_flops": th, "ms_per_step": ms}


def main(argv=None):
    import argparse

    import torch
    ap = argparse.ArgumentParser(prog="python -m mpsb200.autotune")
    ap.add_argument("--out", default=TABLE_PATH)
    ap.add_argument("--copies", type=int, default=16)
    ap.add_argument("--rho-copies", type=int, default=4)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args(argv)
    entries = []
    for chi in TRAJ_CAPS:
        entries.append(tune("trajectory", 64, chi, a.copies, a.steps, a.warmup))
        print(json.dumps(entries[-1]), flush=True)
    for chi in RHO_CAPS:
        entries.append(tune("density", 40, chi, a.rho_copies, a.steps, a.warmup))
        print(json.dumps(entries[-1]), flush=True)
    table = {"device": torch.cuda.get_device_name(0),
             "how": "ms per batched step of one bucket (trajectories: N=64, %d copies, coherent steps; "
                    "density matrices: N=40, %d copies), %d steps after %d warm-up steps per candidate "
                    "(slices, min_flops); the fastest candidate is the entry's choice"
                    % (a.copies, a.rho_copies, a.steps, a.warmup),
             "entries": entries}
    with open(a.out, "w") as f:
        json.dump(table, f, indent=1)
    print(a.out)


if __name__ == "__main__":
    main()
