#!/usr/bin/env python
"""Benchmark of the RK4 MPS/MPO time step (RK4stp_apply_H_half!, src/timeevolution.jl:178-196).

Workload (default, --workload batch): 256 independent quantum trajectories of the driven waveguide
chain (N=64 two-level sites, d=2, exact MPO w=4, dt=0.01, all-down start), bond caps log-uniform
over 8..256 on a 16-value grid, each trajectory its own seeded uniform stream; one step = one
step of the trajectory example loop for every trajectory (examples/spin_model_quantum_trajectory_
rk4.jl:104-209: the RK4 step, the norm, the jump decision, the jump compressions on jump steps).
Measured: the batched engine with the larger contractions on the int8-sliced tensor-core path
(the headline), the same engine in FP64, and the plain FP64 path running the trajectories one
at a time (the drop-in); the p_coh records of split and FP64 are compared step by step.
--workload precision: one density matrix N=60, d=4, chi=512, w=8 from a random chi=64 start,
split path beside FP64, per-step observable errors, the FP64 sensitivity envelope and a
physical-start accuracy check.  --workload density: the plain-FP64 density matrix N=40, chi=128.
Metric: site-updates/s = trajectories x sites x steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload batch|precision|density]
    python bench.py --op qr|gemm-mix|zgemm|rk4 ...        per-operation timing (see run_op)

Our arm: device-resident state, CUDA-event timing of K steps (max over ranks); each rank runs its
own independent replica of the workload (weak scaling).  Reference arm (--impl reference): the
CPU oracle (NumPy/OpenBLAS restatement of the reference's Julia code, which cannot run here) on
the host cores, rank 0 only, on a bounded sample of the workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "matrixproductstates.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOADS = {
    "precision": dict(na=60, d=4, chi=512, chi0=64, seed=60, w=8, dt=0.005, gam_eg=0.1, omega=0.5, gam_phi=0.1,
                      slices=6, pairs=((0, 1), (29, 30), (9, 49)), golden="rho_n60_chi512.npz"),
    "density": dict(na=40, d=4, chi=128, chi0=0, seed=0, w=8, dt=0.005, gam_eg=0.1, omega=0.5, gam_phi=0.1,
                    slices=0, pairs=((0, 1), (9, 10), (19, 20), (4, 34)), golden="rho_n40_chi128.npz"),
    # independent trajectories of the driven waveguide chain (d=2, w=4), per-trajectory bond caps
    # log-uniform over 8..256 on a 16-value grid, every trajectory its own seed
    "batch": dict(na=64, d=2, chi=256, w=4, dt=0.01, omega=0.5, ntraj=256, chi_seed=3, slices=6,
                  grid=[int(round(8 * 32 ** (j / 15.0))) for j in range(16)]),
}
METRIC = "MPS site-updates/s (RK4 step)"
UNIT = "site-updates/s"
# dram__bytes_read.sum + dram__bytes_write.sum of one cluster-QR launch at the chi=128 interior
# shape (512 x 128; the input read once, the outputs stay in L2), from one ncu capture
QR_TRAFFIC_BYTES = 1114624
# dram__bytes_read.sum + dram__bytes_write.sum of one launch of the sliced GEMM's tensor-core
# kernel at M=512, N=2048, K=4096 (6 slices; the chi=512 effective-operator shape), from one ncu
# capture (251.1 MB read + 15.4 MB written); its algorithmic bytes (slices in, C out) are 243 MB
OZ_TRAFFIC_BYTES = 266535168


def dims_rule(na, dmax, d):
    dims = [1] * (na + 1)
    for k in range(1, na):
        dims[k] = dmax
    for n in range(1, na):
        dims[n] = min(dims[n - 1] * d, dims[n])
        dims[na - n] = min(dims[na + 1 - n] * d, dims[na - n])
    return dims


def step_flops(dims, w, d):
    """Algorithmic flops of one RK4 step, counted op by op as the sweeps issue them
    (complex GEMM = 8 M N K; MPO apply = 8 X Y K M; QR = 16 (m n^2 - n^3/3))."""
    na = len(dims) - 1
    f = {"gemm": 0.0, "mpo": 0.0, "qr": 0.0}

    def aor(Dl, Dr, wl, wr):
        f["gemm"] += 8.0 * (Dl * d) * (wr * Dr) * Dr
        f["mpo"] += 8.0 * Dl * Dr * (d * wr) * (wl * d)

    def aol(Dl, Dr, wl, wr):
        f["gemm"] += 8.0 * (wl * Dl) * (d * Dr) * Dl
        f["mpo"] += 8.0 * Dl * Dr * (wl * d) * (d * wr)

    def g(m, n, k):
        f["gemm"] += 8.0 * m * n * k

    def qr(m, n):
        f["qr"] += 16.0 * (m * n * n - n ** 3 / 3.0)

    def stage(right, npl):
        for k in range(na):
            Dl, Dr, wl, wr = dims[k], dims[k + 1], w[k], w[k + 1]
            if not right and k < na - 1:                      # left env init
                for _ in range(npl):
                    g(Dl, d * Dr, Dl); g(Dr, Dr, Dl * d)
                aol(Dl, Dr, wl, wr); g(Dr * wr, Dr, Dl * d)
            if right and k >= 1:                              # right env init
                for _ in range(npl):
                    g(Dl * d, Dr, Dr); g(Dl, Dl, d * Dr)
                aor(Dl, Dr, wl, wr); g(Dl * wl, Dl, d * Dr)
            for _ in range(npl):                              # sweep, plain terms
                g(Dl, d * Dr, Dl); g(Dl * d, Dr, Dr)
            if right:
                aol(Dl, Dr, wl, wr); g(Dl * d, Dr, Dr * wr)
                if k < na - 1:
                    qr(d * Dl, Dr)
                    for _ in range(npl):
                        g(Dr, Dr, Dl * d)
                    g(Dr * wr, Dr, Dl * d)
            else:
                aor(Dl, Dr, wl, wr); g(Dl, d * Dr, Dl * wl)
                if k > 0:
                    qr(d * Dr, Dl)
                    for _ in range(npl):
                        g(Dl, Dl, d * Dr)
                    g(Dl * wl, Dl, d * Dr)

    stage(False, 0)
    stage(True, 1)
    stage(False, 1)
    stage(True, 3)
    return f


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def cpu_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count()


def max_over_ranks(x, dist, device="cuda"):
    """The largest of the ranks' x, on every rank (x itself without a process group): the
    job's time is its slowest replica's."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, sites, steps, secs):
    """Whole-job site-updates/s: every rank evolves its own replica of `sites` sites."""
    return world * sites * steps / secs


def run_serving():
    """p50/p99 job latency of a bounded sample of the mixed serving stream with the configuration's
    size ranges: 24 seeded Poisson arrivals at 200 jobs/s, 70% trajectories (N 20..100, d=2, w=4,
    chi in {32, 64, 128, 256, 512}) and 30% density matrices (N 20..60, d=4, w=8, chi in {64, 128,
    256}), 3..6 RK4 steps each (the configuration's 100..500 would run for many minutes), up to 16
    jobs on the device in shared buckets of the batched engine (continuous batching, 6 int8
    slices for the larger contractions)."""
    from mpsb200 import serve as S
    jobs = S.poisson_jobs(24, 200.0, 11, traj_na=(20, 100), traj_chi=(32, 64, 128, 256, 512), rho_na=(20, 60),
                          rho_chi=(64, 128, 256), steps=(3, 6))
    buckets = {}

    def seen(sl):
        buckets.setdefault(id(sl.bucket), []).append(sl.job.job_id)

    done, st = S.Server(max_jobs=16, slots=8, slices=6).run(jobs, on_admit=seen)
    return {"jobs": st["jobs"], "arrival_rate_per_s": 200.0, "max_running": 16, "mode": "shared buckets",
            "buckets": len(buckets), "jobs_per_bucket_max": max(len(v) for v in buckets.values()),
            "latency_p50_ms": 1e3 * st["latency_p50_s"], "latency_p99_ms": 1e3 * st["latency_p99_s"],
            "queue_p50_ms": 1e3 * st["queue_p50_s"], "site_updates_per_s": st["site_updates_per_s"],
            "wall_s": st["wall_s"], "failed": len(st["failed"]), "refused": len(st["refused"]),
            "sample": "24 jobs: 70% trajectories N 20..100 chi 32..512, 30% rho N 20..60 chi 64..256, 3..6 steps"}


def _event_us(torch, stream, fn, reps, warmup, ctx):
    for _ in range(warmup):
        fn()
    ctx.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    return e0.elapsed_time(e1) * 1e3 / reps


def run_op(argv):
    """Per-operation timing through the C ABI (CUDA events, one GPU), one JSON line; small
    enough to run under a profiler with --reps 1:

        bench.py --op qr M N                     mpsb_op_qr (leftorth!/rightorth!, src/orthonormalisation.jl:164-234)
        bench.py --op gemm-mix [--chi --d --w]   prod_LR (3,4) / (4,3), update_re!, update_le! of one interior site
        bench.py --op zgemm M N K [--slices S]   mpsb_op_zgemm, FP64 (S=0) or int8-sliced tensor-core path
        bench.py --op batch [CHI [T]] [--slices S]  steps of the batching workload (or of T trajectories of
                                                 cap CHI), each inside an NVTX range "batch_step"
        bench.py --op rk4 [N] [--chi --w --slices S --random CHI0]
                                                 in-place RK4 steps of the density-matrix workload, each timed
                                                 step inside an NVTX range "rk4_step"
    """
    ap = argparse.ArgumentParser(prog="bench.py --op")
    ap.add_argument("op", choices=["qr", "gemm-mix", "zgemm", "rk4", "batch"])
    ap.add_argument("dims", nargs="*", type=int)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chi", type=int, default=128)
    ap.add_argument("--d", type=int, default=4)
    ap.add_argument("--w", type=int, default=8)
    ap.add_argument("--slices", type=int, default=0)
    ap.add_argument("--random", type=int, default=0, help="rk4: start from a random MPS of this bond dim")
    a = ap.parse_args(argv)

    import ctypes as C

    import torch

    import __graft_entry__
    __graft_entry__.build()
    import mpsb200 as K
    from mpsb200 import _lib

    ctx = K.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(1234)
    out = {"op": a.op}
    if a.op == "batch":
        import numpy as np
        from mpsb200 import batch as BT, models as GM
        W = WORKLOADS["batch"]
        chis = batch_chis(W) if not a.dims else [a.dims[0]] * (a.dims[1] if len(a.dims) > 1 else 16)
        n = a.warmup + a.reps
        u = [_uniforms(k, n) for k in range(len(chis))]
        tb = BT.TrajectoryBatch(GM.WaveguideChain(W["na"], omega=W["omega"]), chis, W["dt"],
                                np.array([x[0] for x in u]), np.array([x[1] for x in u]), slices=a.slices)
        for _ in range(a.warmup):
            tb.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.reps):
            torch.cuda.nvtx.range_push("batch_step")
            tb.step()
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        ms = (time.perf_counter() - t0) * 1e3 / a.reps
        tb.close()
        out.update({"trajectories": len(chis), "slices": a.slices, "ms_per_step": ms,
                    "site_updates_per_s": W["na"] * len(chis) / ms * 1e3})
    elif a.op == "qr":
        m, n = a.dims[:2] if len(a.dims) >= 2 else (512, 128)
        X = torch.randn(m * n, dtype=torch.complex128, device="cuda", generator=g)
        Q = torch.empty_like(X)
        torch.cuda.synchronize()
        args = (C.c_void_p(X.data_ptr()), C.c_void_p(Q.data_ptr()), None, m, n)
        us = _event_us(torch, stream, lambda: _lib.call("mpsb_op_qr", ctx.h, *args), a.reps, a.warmup, ctx)
        flops = 16.0 * (m * n * n - n ** 3 / 3.0)   # factorisation + forming Q (complex)
        out.update({"m": m, "n": n, "us": us, "tflops": flops / us / 1e6})
    elif a.op == "zgemm":
        M, N, Kd = a.dims[:3] if len(a.dims) >= 3 else (512, 2048, 4096)
        A = torch.randn(M * Kd, dtype=torch.complex128, device="cuda", generator=g)
        B = torch.randn(Kd * N, dtype=torch.complex128, device="cuda", generator=g)
        Cm = torch.zeros(M * N, dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        args = (ctx.h, M, N, Kd, C.c_void_p(A.data_ptr()), 1, M, 1, C.c_void_p(B.data_ptr()), 1, Kd, 0,
                C.c_void_p(Cm.data_ptr()), 1, M, None, None, a.slices)
        us = _event_us(torch, stream, lambda: _lib.call("mpsb_op_zgemm", *args), a.reps, a.warmup, ctx)
        out.update({"M": M, "N": N, "K": Kd, "slices": a.slices, "us": us, "tflops": 8.0 * M * N * Kd / us / 1e6})
    elif a.op == "rk4":
        from mpsb200 import drivers as GDR, models as GM
        na = a.dims[0] if a.dims else 40
        ctx.set_precision(a.slices)
        p = GM.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
        rho = None
        if a.random:
            import numpy as np
            rho, _ = K.mpsrandom(na, a.random, 4, np.random.default_rng(60), ctx)
            K.normalize_lo_(rho)
            rho, _ = K.expandmps(rho, a.chi, ctx)
        b = GDR.DensityBuffers(p, a.chi, 0.005, a.w, ctx, rho)
        for _ in range(a.warmup):
            b.step()
        ctx.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.reps):
            torch.cuda.nvtx.range_push("rk4_step")
            b.step()
            torch.cuda.nvtx.range_pop()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.sync()
        ms = e0.elapsed_time(e1) / a.reps
        out.update({"na": na, "chi": a.chi, "w": a.w, "slices": a.slices, "random_start": a.random,
                    "ms_per_step": ms, "site_updates_per_s": na / ms * 1e3})
    else:
        chi, d, w = a.chi, a.d, a.w
        bufs = [torch.randn(chi * w * d * chi, dtype=torch.complex128, device="cuda", generator=g) for _ in range(3)]
        torch.cuda.synchronize()
        p = [C.c_void_p(b.data_ptr()) for b in bufs]
        calls = [
            ("prod_LR_3_4", "mpsb_op_prod_LR_3_4", (p[0], p[1], p[2], chi, w, chi, d, chi)),
            ("update_re", "mpsb_op_update_re", (p[2], p[1], p[0], chi, w, d, chi, chi)),
            ("prod_LR_4_3", "mpsb_op_prod_LR_4_3", (p[0], p[1], p[2], chi, d, chi, w, chi)),
            ("update_le", "mpsb_op_update_le", (p[2], p[0], p[1], chi, d, chi, w, chi)),
        ]
        flops = 8.0 * w * d * chi ** 3
        tot = 0.0
        for tag, name, args in calls:
            us = _event_us(torch, stream, lambda: _lib.call(name, ctx.h, *args), a.reps, a.warmup, ctx)
            out[tag] = {"us": us, "tflops": flops / us / 1e6}
            tot += us
        out.update({"chi": chi, "d": d, "w": w, "mix_us": tot, "mix_tflops": 4 * flops / tot / 1e6})
    ctx.close()
    print(json.dumps(out), flush=True)


def load_peaks():
    """(int8 dense TOP/s, source) for the sliced GEMM's roofline: twice the measured dense bf16
    rate of MEASURED_PEAKS.json (the int8 kind runs the same tensor pipe at twice the bf16
    rate), else twice the pool's fallback bf16 figure."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        bf16 = float(pk.get("bf16_tflops"))
        return 2.0 * bf16, "2 x bf16_tflops %.1f of measured (MEASURED_PEAKS.json)" % bf16
    except Exception:
        return 2.0 * 1590.0, "2 x 1590 TFLOP/s bf16 of fallback (no MEASURED_PEAKS.json)"


def workload_buffers(W, ctx, slices, start=None, perturb=0.0):
    """Device buffers of the workload's density matrix on ctx, contractions at `slices`; start
    "random" (chi0 > 0) or "down" (all-down product), every site entry scaled by
    (1 + perturb N(0,1)) when perturb > 0."""
    import numpy as np

    import mpsb200 as K
    from mpsb200 import drivers as GDR
    from mpsb200 import models as GM
    ctx.set_precision(slices)
    p = GM.WaveguideChain(W["na"], gam_eg=W["gam_eg"], omega=W["omega"], gam_phi=W["gam_phi"])
    if start is None:
        start = "random" if W["chi0"] else "down"
    rho = None
    if start == "random":
        rho, _ = K.mpsrandom(W["na"], W["chi0"], W["d"], np.random.default_rng(W["seed"]), ctx)
        K.normalize_lo_(rho)
        rho, _ = K.expandmps(rho, W["chi"], ctx)
    elif perturb:
        rho, _ = K.mpsgroundstate(W["na"], W["chi"], W["d"], ctx)
    if perturb:
        rng = np.random.default_rng(5)
        for k in range(rho.na):
            s = rho.site(k)
            rho.set_site(k, s * (1 + perturb * rng.standard_normal(s.shape)))
    return GDR.DensityBuffers(p, W["chi"], W["dt"], W["w"], ctx, rho), p


def accuracy_arms(W, steps, local_rank):
    """The split path against FP64 where the comparison is meaningful: (1) the FP64 path from the random
    start perturbed by 1e-15 relative (the sensitivity of the truncated dynamics to rounding:
    any two FP64 implementations differ by this much), (2) split and FP64 from the physical
    all-down start at the same sizes, observables after every step."""
    import mpsb200 as K
    pairs = W["pairs"]
    out = {}

    def run(slices, start, perturb=0.0):
        c = K.Context(local_rank)
        try:
            b, _ = workload_buffers(W, c, slices, start, perturb)
            recs = []
            for _ in range(steps):
                b.step()
                recs.append(b.observables(pairs))
            c.sync()
            del b
        finally:
            c.close()
        return recs
    if W["chi0"]:
        ref = run(0, "random")
        pert = run(0, "random", 1e-15)
        out["fp64_envelope_rel_per_step"] = [e / s for e, s in (obs_error(a, b) for a, b in zip(pert, ref))]
    d64 = run(0, "down")
    dsp = run(W["slices"], "down")
    out["down_start_obs_err_per_step_vs_fp64"] = [obs_error(a, b)[0] for a, b in zip(dsp, d64)]
    out["down_start_trace_rho"] = [float(abs(r[0])) for r in d64]
    return out


def obs_error(a, b):
    """max |difference| of two (Tr rho, <see_i>, <s+_i s-_j>) records and the records' scale"""
    import numpy as np
    err = max(abs(a[0] - b[0]), float(np.abs(np.asarray(a[1]) - np.asarray(b[1])).max()),
              float(np.abs(np.asarray(a[2]) - np.asarray(b[2])).max()))
    scale = max(abs(b[0]), float(np.abs(np.asarray(b[1])).max()), float(np.abs(np.asarray(b[2])).max()))
    return err, scale


def oracle_site_sample(W, threads_note=""):
    """One interior site-update on the CPU oracle: every contraction and QR that an interior site
    (chi x d x chi, MPO bonds w) undergoes in the four stages of one RK4 step, in the sweeps'
    order (environment initialisation, plain terms, the operator term, the QR, environment
    updates), on seeded random tensors.  Returns (seconds, algorithmic flops of the sample)."""
    import numpy as np

    from oracle import mps_ref as R
    chi, d, w = W["chi"], W["d"], W["w"]
    rng = np.random.default_rng(1)

    def cr(*s):
        return (rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex128)
    A, A0 = cr(chi, d, chi), cr(chi, d, chi)
    O = cr(w, d, w, d)
    F3L, F3R = cr(chi, w, chi), cr(chi, w, chi)
    F2 = cr(chi, chi)
    flops = [0.0]

    def g(m, n, k):
        flops[0] += 8.0 * m * n * k
    t0 = time.perf_counter()
    for right, npl in ((False, 0), (True, 1), (False, 1), (True, 3)):
        for _ in range(npl):                      # environment initialisation, plain terms
            if right:
                AR = R.prod_LR(A, F2); g(chi * d, chi, chi)
                R.update_renv(A0, AR); g(chi, chi, d * chi)
            else:
                AL = R.prod_LR(F2, A); g(chi, d * chi, chi)
                R.update_lenv(A0, AL); g(chi, chi, chi * d)
        if right:                                 # environment initialisation, operator term
            T = R.prod_AOR(A, O, F3R); g(chi * d, w * chi, chi); flops[0] += 8.0 * chi * chi * d * w * w * d
            R.update_re(A0, T); g(chi * w, chi, d * chi)
        else:
            T = R.prod_AOL(A, O, F3L); g(w * chi, d * chi, chi); flops[0] += 8.0 * chi * chi * d * w * w * d
            R.update_le(A0, T); g(chi * w, chi, chi * d)
        for _ in range(npl):                      # the sweep: plain terms
            P = R.prod_LR(F2, A); g(chi, d * chi, chi)
            R.prod_LR(P, F2); g(chi * d, chi, chi)
        if right:                                 # operator term, QR, environment updates
            T = R.prod_AOL(A, O, F3L); g(w * chi, d * chi, chi); flops[0] += 8.0 * chi * chi * d * w * w * d
            B = R.prod_LR(T, F3R); g(chi * d, chi, chi * w)
            Q = R.leftorth_(B); flops[0] += 16.0 * (d * chi * chi * chi - chi ** 3 / 3.0)
            for _ in range(npl):
                R.update_lenv(Q, P); g(chi, chi, chi * d)
            R.update_le(Q, T); g(chi * w, chi, chi * d)
        else:
            T = R.prod_AOR(A, O, F3R); g(chi * d, w * chi, chi); flops[0] += 8.0 * chi * chi * d * w * w * d
            B = R.prod_LR(F3L, T); g(chi, d * chi, chi * w)
            Q = R.rightorth_(B); flops[0] += 16.0 * (d * chi * chi * chi - chi ** 3 / 3.0)
            for _ in range(npl):
                R.update_renv(Q, P); g(chi, chi, d * chi)
            R.update_re(Q, T); g(chi * w, chi, d * chi)
    return time.perf_counter() - t0, flops[0]


def cpu_rate(W, nsamples):
    """Chain-average site-updates/s of the CPU oracle: interior site-update samples scaled by
    the flop model's ratio of the interior site to the chain's mean site."""
    dims = dims_rule(W["na"], W["chi"], W["d"])
    wv = [1] + [W["w"]] * (W["na"] - 1) + [1]
    mean_site = sum(step_flops(dims, wv, W["d"]).values()) / W["na"]
    times, fl = [], 0.0
    for _ in range(nsamples):
        t, fl = oracle_site_sample(W)
        times.append(t)
    tot = sum(times)
    return nsamples * (fl / mean_site) / tot, tot / nsamples, fl, mean_site


def batch_chis(W):
    """Per-trajectory bond caps: u_k ~ U[0,1) (seeded), chi_k = the grid value nearest to 8*32^u_k
    on the log scale."""
    import numpy as np
    u = np.random.default_rng(W["chi_seed"]).random(W["ntraj"])
    g = np.log(np.array(W["grid"], dtype=float))
    return [W["grid"][int(np.argmin(np.abs(g - np.log(8 * 32 ** x))))] for x in u]


def batch_flops(W, chis):
    """Algorithmic flops of one step of every trajectory: the RK4 step of step_flops plus the
    two jump compressions (one R->L and one L->R sweep with the w=2 jump MPO, compress_var_apply_H!
    with maxsweeps = 1 after its environment initialisation)."""
    tot = 0.0
    for c in set(chis):
        n = chis.count(c)
        dims = dims_rule(W["na"], c, W["d"])
        wv = [1] + [W["w"]] * (W["na"] - 1) + [1]
        f = sum(step_flops(dims, wv, W["d"]).values())
        wj = [1] + [2] * (W["na"] - 1) + [1]
        fj = step_flops_jump(dims, wj, W["d"])
        tot += n * (f + 2 * fj)
    return tot


def step_flops_jump(dims, w, d):
    """flops of compress_var_apply_H!(A0, envop, A, A, H, 1): left env init, one R->L and one
    L->R sweep (prod_AOR/AOL, prod_LR, QR, env update per site)."""
    na = len(dims) - 1
    f = 0.0
    for k in range(na):
        Dl, Dr, wl, wr = dims[k], dims[k + 1], w[k], w[k + 1]
        aol = 8.0 * (wl * Dl) * (d * Dr) * Dl + 8.0 * Dl * Dr * (wl * d) * (d * wr)
        aor = 8.0 * (Dl * d) * (wr * Dr) * Dr + 8.0 * Dl * Dr * (d * wr) * (wl * d)
        if k < na - 1:
            f += aol + 8.0 * (Dr * wr) * Dr * (Dl * d)                                  # init
            f += aol + 8.0 * (Dl * d) * Dr * (Dr * wr) + 16.0 * ((d * Dl) * Dr * Dr - Dr ** 3 / 3.0) \
                + 8.0 * (Dr * wr) * Dr * (Dl * d)                                       # L->R sweep
        else:
            f += aol + 8.0 * (Dl * d) * Dr * (Dr * wr)
        if k > 0:
            f += aor + 8.0 * Dl * (d * Dr) * (Dl * wl) + 16.0 * ((d * Dr) * Dl * Dl - Dl ** 3 / 3.0) \
                + 8.0 * (Dl * wl) * Dl * (d * Dr)                                       # R->L sweep
    return f


def config_dict(args, W):
    if args.workload == "batch":
        return {"workload": "%d independent quantum trajectories of the driven waveguide chain N=%d, d=2, w=4, "
                            "dt=%g, bond caps log-uniform 8..256 (16-value grid), all-down start; one step = the "
                            "example loop's step of every trajectory (RK4 step, both jump compressions, norms, "
                            "jump decisions); contractions int8-sliced x%d on tcgen05 (the larger ones), QR / "
                            "norms FP64" % (W["ntraj"], W["na"], W["dt"], W["slices"]),
                "name": "batch", "trajectories": W["ntraj"], "sites": W["na"], "d": 2, "w": 4, "dt": W["dt"],
                "chi_grid": W["grid"], "slices": W["slices"],
                "parallelism": "replicas x%d; trajectories grouped in per-chi buckets, one stream each" % args.gpus,
                "l2": "working set per step > 126 MB L2 (no flush needed)"}
    return {"workload": "density-matrix RK4 step, waveguide spin chain N=%d, d=%d, chi=%d, w=%d (6 + 2 zero "
                        "channels), dt=%g, %s start%s" % (
                            W["na"], W["d"], W["chi"], W["w"], W["dt"],
                            ("random chi=%d (seed %d) zero-padded" % (W["chi0"], W["seed"])) if W["chi0"]
                            else "all-down product",
                            (", contractions int8-sliced x%d on tcgen05, QR/norms FP64" % W["slices"])
                            if W["slices"] else ", FP64"),
            "name": args.workload, "sites": W["na"], "d": W["d"], "chi": W["chi"], "w": W["w"], "dt": W["dt"],
            "slices": W["slices"],
            "parallelism": "replicas x%d (independent rho per GPU)" % args.gpus,
            "l2": "working set per step > 126 MB L2 (no flush needed)"}


def run_reference(args, rank):
    if rank != 0:
        return None
    W = WORKLOADS[args.workload]
    if args.workload == "batch":
        chis = batch_chis(W)
        model, cores = cpu_info()
        cb = None
        vals = []
        for _ in range(max(1, args.steps)):
            cb = batch_cpu_baseline(W, chis)
            vals.append(cb["value"])
        value = sum(vals) / len(vals)
        cb["value"] = value
        return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": 0, "ms_per_step": 1e3 * W["na"] * W["ntraj"] / value,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
                "data": "synthetic (all-down trajectories)", "config": config_dict(args, W), "cpu_baseline": cb,
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    model, cores = cpu_info()
    for _ in range(args.warmup):
        oracle_site_sample(W)
    value, t_sample, fl, mean_site = cpu_rate(W, args.steps)
    sample = ("%d interior site-updates (chi=%d, d=%d, w=%d: all contractions and the QR of one site in the "
              "four stages of an RK4 step) on the CPU oracle (NumPy/OpenBLAS, %s, %d threads), %.2f s each; "
              "chain-average rate = interior rate x interior/mean site flops (%.3g/%.3g)"
              % (args.steps, W["chi"], W["d"], W["w"], model, cores, t_sample, fl, mean_site))
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * W["na"] / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic (seeded random tensors of the workload's interior shapes)",
        "config": config_dict(args, W),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def time_qr(ctx, torch, stream, m, n):
    """CUDA-event timing of one QR of the interior-site shape (d*chi x chi) through the op API:
    returns (algorithmic flops, seconds) per QR."""
    import ctypes as C
    from mpsb200 import _lib
    g = torch.Generator(device="cuda").manual_seed(7)
    X = torch.randn(m * n, dtype=torch.complex128, device="cuda", generator=g)
    Q = torch.empty_like(X)
    torch.cuda.synchronize()
    args = (C.c_void_p(X.data_ptr()), C.c_void_p(Q.data_ptr()), None, m, n)
    us = _event_us(torch, stream, lambda: _lib.call("mpsb_op_qr", ctx.h, *args), 5, 2, ctx)
    del X, Q
    return 16.0 * (m * n * n - n ** 3 / 3.0), us * 1e-6


def time_sliced_gemm(ctx, torch, stream, W):
    """CUDA-event device time of the tensor-core kernel of the sliced GEMM at the workload's
    effective-operator shape (prod_LR 3-index: M=chi, N=d chi, K=w chi), read through the
    context's profiling hook, and of the whole sliced GEMM (slicing kernels included)."""
    import ctypes as C
    from mpsb200 import _lib
    S, chi, d, w = W["slices"], W["chi"], W["d"], W["w"]
    M, N, Kd = chi, d * chi, w * chi
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(M * Kd, dtype=torch.complex128, device="cuda", generator=g)
    B = torch.randn(Kd * N, dtype=torch.complex128, device="cuda", generator=g)
    Cm = torch.zeros(M * N, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    args = (ctx.h, M, N, Kd, C.c_void_p(A.data_ptr()), 1, M, 1, C.c_void_p(B.data_ptr()), 1, Kd, 0,
            C.c_void_p(Cm.data_ptr()), 1, M, None, None, S)
    reps = 10
    us_all = _event_us(torch, stream, lambda: _lib.call("mpsb_op_zgemm", *args), reps, 2, ctx)
    ctx.profile_read()
    ctx.set_profiling(True)
    for _ in range(reps):
        _lib.call("mpsb_op_zgemm", *args)
    ms, n, _ = ctx.profile_read()
    ctx.set_profiling(False)
    del A, B, Cm
    int8_ops = 2.0 * (S * (S + 1) // 2) * M * (2 * N) * (2 * Kd)
    return {"M": M, "N": N, "K": Kd, "slices": S, "kernel_us": 1e3 * ms / n, "op_us": us_all,
            "int8_ops": int8_ops, "complex_flops": 8.0 * M * N * Kd}


def run_ours(args, rank, world, local_rank, dist):
    import ctypes as C

    import numpy as np
    import torch

    import mpsb200 as K
    from mpsb200 import _lib
    from mpsb200 import models as GM

    torch.cuda.set_device(local_rank)
    W = WORKLOADS[args.workload]
    pairs = W["pairs"]
    split = W["slices"] > 0
    ctx = K.Context(local_rank)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    b, p = workload_buffers(W, ctx, W["slices"])
    dims = b.dims
    wv = [1] + [W["w"]] * (W["na"] - 1) + [1]
    fl = step_flops(dims, wv, W["d"])

    # ---- warm-up of the measured arm, observables after every step
    obs0 = b.observables(pairs)
    obs = []
    for _ in range(args.warmup):
        b.step()
        obs.append(b.observables(pairs))
    ctx.sync()

    # ---- the plain FP64 path on the same start, warm-up steps with observables
    fp = None
    if split:
        ctx64 = K.Context(local_rank)
        stream64 = torch.cuda.Stream()
        ctx64.set_stream(stream64.cuda_stream)
        b64, _ = workload_buffers(W, ctx64, 0)
        obs64 = []
        for _ in range(args.warmup):
            b64.step()
            obs64.append(b64.observables(pairs))
        ctx64.sync()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    l0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        torch.cuda.nvtx.range_push("rk4_step")
        b.step()
        torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = ctx.launches - l0
    secs = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
    value = job_rate(world, W["na"], args.steps, secs)
    obs_end = b.observables(pairs)

    check = {"trace_rho_end": float(np.real(obs_end[0])), "steps_compared": args.warmup}
    if split:
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream64)
        for _ in range(args.steps):
            b64.step()
        f1.record(stream64)
        torch.cuda.synchronize()
        secs64 = max_over_ranks(f0.elapsed_time(f1) / 1e3, dist)
        value64 = job_rate(world, W["na"], args.steps, secs64)
        obs64_end = b64.observables(pairs)
        per_step = [obs_error(o, r) for o, r in zip(obs, obs64)]
        err_end, scale_end = obs_error(obs_end, obs64_end)
        ab = K.scal_prod(b.rho, b64.rho)
        fid = abs(ab) ** 2 / (K.scal_prod(b.rho, b.rho).real * K.scal_prod(b64.rho, b64.rho).real)
        del b64
        ctx64.close()
        fp = {"value": value64, "ms_per_step": 1e3 * secs64 / args.steps,
              "split_vs_fp64": value / value64}
        check.update({"obs_err_per_step_vs_fp64": [e for e, _ in per_step],
                      "obs_scale": max(s for _, s in per_step) if per_step else None,
                      "obs_rel_err_max_vs_fp64": max((e / s for e, s in per_step), default=None),
                      "obs_err_after_%d_steps_vs_fp64" % (args.warmup + args.steps): err_end,
                      "obs_rel_err_after_%d_steps_vs_fp64" % (args.warmup + args.steps): err_end / scale_end,
                      "infidelity_vs_fp64_after_%d_steps" % (args.warmup + args.steps): 1.0 - fid})
    # oracle golden values of the first steps (tests/golden), when present
    gpath = os.path.join(ROOT, "tests", "golden", W["golden"])
    if os.path.exists(gpath):
        gz = np.load(gpath)
        mi = 1 if W["chi0"] else 10      # steps between the fixture's records
        recs = [obs0] + obs              # the measured arm after 0..warmup steps
        errs = [obs_error(recs[i], (gz["tr"][i // mi], gz["see"][i // mi], gz["spm"][i // mi]))
                for i in range(0, len(recs), mi) if i // mi < len(gz["tr"])]
        if errs:
            check["obs_rel_err_vs_oracle_golden"] = max(e / s for e, s in errs)
            check["golden_steps"] = len(errs) - 1

    # ---- end to end through the public API with host buffers: every step uploads the three
    # generator MPOs from pinned host memory (the reference loop's update_L! refresh) and reads
    # Tr(rho) back (the measurement of the example loop)
    mpo_host = []
    h2d = 0
    for (con, delt, tt) in [(1, W["dt"] / 2, 0.0), (0, 1, W["dt"] / 2), (1, W["dt"] / 2, W["dt"])]:
        sites = GM.construct_L_spin_model(p, con, delt, tt, W["w"])
        pinned = []
        for s in sites:
            pt = torch.empty(s.size * 2, dtype=torch.float64, pin_memory=True)
            arr = pt.numpy()
            arr[:] = np.ascontiguousarray(s.ravel(order="F")).view(np.float64)
            pinned.append((pt, arr.reshape(-1)))
            h2d += s.size * 16
        mpo_host.append(pinned)
    ke = max(2, args.steps)

    def e2e_step():
        for mpo, pinned in zip(b.L, mpo_host):
            for k, (_, arr) in enumerate(pinned):
                _lib.call("mpsb_mpo_set_site", mpo.h, k + 1, arr.ctypes.data_as(C.POINTER(C.c_double)))
        b.step()
        K.scal_prod_no_conj(b.trace_fn, b.rho)

    for _ in range(min(args.warmup, 2)):
        e2e_step()
    ctx.sync()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        e2e_step()
    ctx.sync()
    e2e_secs = max_over_ranks(time.perf_counter() - t0, dist)
    e2e_value = job_rate(world, W["na"], ke, e2e_secs)

    # ---- roofline of the dominant kernel
    if split:
        peak, src = load_peaks()
        sg = time_sliced_gemm(ctx, torch, stream, W)
        ach = sg["int8_ops"] / sg["kernel_us"] / 1e6
        roofline = {"bound": "tensor", "pipe": "int8 (tcgen05 kind::i8)", "kernel": "ozgemm_kernel<%d>" % W["slices"],
                    "achieved": ach, "peak": peak, "unit": "TOP/s", "frac": ach / peak, "peak_source": src,
                    "traffic": OZ_TRAFFIC_BYTES if (sg["M"], sg["N"], sg["K"], W["slices"]) == (512, 2048, 4096, 6) else None,
                    "per_launch": "prod_LR 3-index shape M=%d N=%d K=%d: %d slice products x 2*M*2N*2K = %.3e int8 "
                                  "ops in %.1f us (CUDA events around the kernel); whole sliced GEMM incl. slicing "
                                  "%.1f us = %.1f complex TFLOP/s" % (
                                      sg["M"], sg["N"], sg["K"], W["slices"] * (W["slices"] + 1) // 2,
                                      sg["int8_ops"], sg["kernel_us"], sg["op_us"],
                                      sg["complex_flops"] / sg["op_us"] / 1e6)}
    else:
        roofline = None
    qm, qn = W["d"] * W["chi"], W["chi"]
    qflops, qsecs = time_qr(ctx, torch, stream, qm, qn)
    roofline_qr = {"bound": "fp64", "kernel": "qr_kernel (cluster Householder) + Q formation",
                   "achieved": qflops / qsecs / 1e12, "unit": "TFLOP/s",
                   "per_launch": "one QR of %d x %d: 16(mn^2 - n^3/3) = %.3e flops in %.1f us"
                                 % (qm, qn, qflops, qsecs * 1e6)}
    if roofline is None:
        roofline = dict(roofline_qr, peak=None, frac=None, traffic=QR_TRAFFIC_BYTES if W["chi"] == 128 else None)

    if split and not args.no_accuracy:
        check.update(accuracy_arms(W, args.warmup, local_rank))
    serving = None
    if world == 1 and not args.no_serve:
        serving = run_serving()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("complex128 operands, int8 slices x%d on the tensor pipe, FP64 QR/norms" % W["slices"]) if split
        else "complex128",
        "data": "synthetic (seeded random / all-down rho, waveguide Lindbladian)",
        "config": config_dict(args, W),
        "clocks": clocks,
        "gpu_launches": int(launches),
        "step_tflops": sum(fl.values()) * args.steps / secs * world / 1e12,
        "step_flops": fl,
        "fp64_path": fp,
        "roofline": roofline,
        "roofline_qr": roofline_qr,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 16,
                "steps": ke},
        "check": check,
        "serving": serving,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        model, cores = cpu_info()
        value_cpu, t_sample, flx, mean_site = cpu_rate(W, 1)
        line["cpu_baseline"] = {"value": value_cpu, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": "1 interior site-update (all its contractions and QRs in one RK4 step, "
                                          "chi=%d) on the CPU oracle (NumPy/OpenBLAS, %s, %d threads): %.2f s; "
                                          "chain rate scaled by interior/mean site flops (%.3g/%.3g)"
                                          % (W["chi"], model, cores, t_sample, flx, mean_site)}
    ctx.close()
    return line


def _uniforms(seed, n):
    import numpy as np
    g = np.random.default_rng(seed)
    return g.random(n), g.random(n)


def run_batch(args, rank, world, local_rank, dist):
    """The batching workload: every trajectory's step through the bucketed batch engine, split
    precision (the headline), beside the same engine in FP64 and the plain FP64 path that runs
    one trajectory at a time (the drop-in, as the reference runs one trajectory per process)."""
    import numpy as np
    import torch

    import mpsb200 as K
    from mpsb200 import batch as BT
    from mpsb200 import drivers as GDR
    from mpsb200 import models as GM

    torch.cuda.set_device(local_rank)
    W = WORKLOADS["batch"]
    chis = batch_chis(W)
    n = args.warmup + args.steps + 1      # + the profiled step
    unif = [_uniforms(1000003 * rank + k, n) for k in range(W["ntraj"])]
    r1 = np.array([u[0] for u in unif])
    r2 = np.array([u[1] for u in unif])
    p = GM.WaveguideChain(W["na"], omega=W["omega"])
    flops_step = batch_flops(W, chis)

    def timed(slices, sample_clocks=False, profile=False, e2e=False):
        # the sliced arms take the autotuner's per-bucket choice (mpsb200/tuning_b200.json)
        tb = BT.TrajectoryBatch(p, chis, W["dt"], r1, r2, device=local_rank, slices=slices, tuned=slices > 0)
        if e2e:   # the example loop: the step's generators uploaded from host memory every step
            host = [tb.generator_sites(i * W["dt"]) for i in range(n)]
            run = lambda i: tb.step(host[i])   # noqa: E731
        else:
            run = lambda i: tb.step()   # noqa: E731
        for i in range(args.warmup):
            run(i)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        sampler = ClockSampler(local_rank) if sample_clocks else None
        if sampler:
            sampler.start()
        l0 = sum(bk.ctx.launches for bk in tb.buckets.values())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for i in range(args.warmup, args.warmup + args.steps):
            run(i)
        torch.cuda.synchronize()
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        clocks = sampler.stop() if sampler else None
        launches = sum(bk.ctx.launches for bk in tb.buckets.values()) - l0
        secs = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
        prof = None
        if profile:   # one more step with the tensor-core kernel bracketed by events
            for bk in tb.buckets.values():
                bk.ctx.set_graphs(False)
                bk.ctx.set_profiling(True)
                bk.ctx.profile_read()
            tb.step()
            ms = ops = cnt = 0.0
            for bk in tb.buckets.values():
                a, c_, o = bk.ctx.profile_read()
                ms, cnt, ops = ms + a, cnt + c_, ops + o
                bk.ctx.set_profiling(False)
            prof = (ms, cnt, ops)
        recs = [tb.records(k)[:2] for k in range(W["ntraj"])]
        h2d = (sum(int(x.nbytes) for x in host[0][0] + host[0][1] + host[0][2]) * len(tb.buckets)) if e2e else 0
        tb.close()
        return secs, wall, launches, clocks, recs, prof, h2d

    secs, wall, launches, clocks, recs, prof, _ = timed(W["slices"], sample_clocks=True, profile=True)
    value = job_rate(world, W["na"] * W["ntraj"], args.steps, secs)
    _, wall_e2e, _, _, _, _, h2d = timed(W["slices"], e2e=True)
    secs64, _, _, _, recs64, _, _ = timed(0)
    value64 = job_rate(world, W["na"] * W["ntraj"], args.steps, secs64)
    dp = max(float(np.abs(np.asarray(a[0])[:len(b[0])] - np.asarray(b[0])).max()) for a, b in zip(recs, recs64))
    nb = args.warmup + args.steps
    same_jumps = sum(1 for a, b in zip(recs, recs64)
                     if [j[:3] for j in a[1] if j[0] < nb] == [j[:3] for j in b[1] if j[0] < nb])
    njumps = sum(len(a[1]) for a in recs)

    # the plain FP64 path, one trajectory at a time: per distinct cap, one trajectory's step time
    plain_t = {}
    for c in sorted(set(chis)):
        ctx = K.Context(local_rank)
        b = GDR.TrajectoryBuffers(p, c, W["dt"], ctx)
        rec = {"p_coh": [], "jumps": []}
        for i in range(n):
            if i == 1:
                ctx.sync()
                t0 = time.perf_counter()
            pc = b.coherent_step()
            GDR.trajectory_decision(b, i, pc, r1[0], r2[0], rec)
        ctx.sync()
        plain_t[c] = (time.perf_counter() - t0) / (n - 1)
        del b
        ctx.close()
    plain_secs = sum(plain_t[c] for c in chis)   # one step of every trajectory, one after the other
    value_plain = job_rate(world, W["na"] * W["ntraj"], 1, plain_secs)

    peak, src = load_peaks()
    ms, cnt, ops = prof
    ach = ops / (ms * 1e-3) / 1e12 if ms > 0 else None
    roofline = {"bound": "tensor", "pipe": "int8 (tcgen05 kind::i8)", "kernel": "ozgemm_kernel<%d>" % W["slices"],
                "achieved": ach, "peak": peak, "unit": "TOP/s", "frac": ach / peak if ach else None,
                "peak_source": src, "traffic": None,
                "traffic_note": "launches of many shapes, no single per-launch figure; at the chi=512 effective-operator "
                                "shape one launch moves %d DRAM bytes (ncu) against 243 MB algorithmic" % OZ_TRAFFIC_BYTES,
                "per_launch": "all %d launches of one step of the workload (every bucket, CUDA events around each "
                              "launch): %.3e int8 ops in %.2f ms" % (cnt, ops, ms)}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "complex128 operands, int8 slices x%d on the tensor pipe for the larger contractions, FP64 "
                 "QR/norms/jump probabilities" % W["slices"],
        "data": "synthetic (all-down trajectories, seeded uniforms, waveguide H)",
        "config": config_dict(args, W), "clocks": clocks, "gpu_launches": int(launches),
        "step_tflops": flops_step * args.steps / secs * world / 1e12,
        "fp64_batched": {"value": value64, "ms_per_step": 1e3 * secs64 / args.steps, "split_vs_fp64_batched": value / value64},
        "fp64_plain_one_at_a_time": {"value": value_plain, "s_per_step_all_trajectories": plain_secs,
                                     "per_chi_s_per_step": plain_t,
                                     "split_batched_vs_plain": value / value_plain},
        "roofline": roofline,
        "e2e": {"value": job_rate(world, W["na"] * W["ntraj"], args.steps, max_over_ranks(wall_e2e, dist)),
                "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8 * W["ntraj"],
                "note": "wall clock of the public API loop (TrajectoryBatch.step): every step uploads the three "
                        "generator MPOs of every bucket from host memory and reads every trajectory's norm back "
                        "for its jump decision (plus the jump norms on jump steps)"},
        "check": {"p_coh_max_abs_err_split_vs_fp64": dp, "trajectories_same_jump_record": same_jumps,
                  "trajectories": W["ntraj"], "jumps": njumps},
    }
    if world == 1 and not args.no_serve:
        line["serving"] = run_serving()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = batch_cpu_baseline(W, chis)
    return line


def batch_cpu_baseline(W, chis, grid=None):
    """CPU oracle on the batching workload: one coherent step (no jump) of one trajectory per
    distinct cap of the sample, timed; the mix's rate = trajectories x sites / sum of their times."""
    import numpy as np

    from oracle import drivers as ODR
    from oracle import models as OM
    model, cores = cpu_info()
    t = {}
    for c in sorted(set(chis) if grid is None else grid):
        p = OM.SpinChain(W["na"], omega=W["omega"])
        t0 = time.perf_counter()
        ODR.run_trajectory(p, c, W["dt"], 1, np.zeros(1), np.zeros(1), measure_int=10)
        t[c] = time.perf_counter() - t0
    tot = sum(t[c] for c in chis)
    value = W["na"] * len(chis) / tot
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "one RK4 step (no jump) of one trajectory per distinct bond cap (%d caps) on the CPU oracle "
                      "(NumPy/OpenBLAS, %s, %d threads), weighted by the caps' counts; %.1f s for the sample"
                      % (len(t), model, cores, sum(t.values()))}


def main():
    if "--op" in sys.argv:
        i = sys.argv.index("--op")
        return run_op(sys.argv[i + 1:])
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream sample")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the envelope / physical-start arms")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_
        torch.cuda.set_device(local_rank)
        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_
    if rank == 0:
        import __graft_entry__
        __graft_entry__.build()   # no-op when libmpsb200.so is current
    if dist:
        dist.barrier()
    if args.workload == "batch":
        line = run_batch(args, rank, world, local_rank, dist)
    else:
        line = run_ours(args, rank, world, local_rank, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
