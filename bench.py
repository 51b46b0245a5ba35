#!/usr/bin/env python
"""Benchmark of the RK4 MPS/MPO time step (RK4stp_apply_H_half!, src/timeevolution.jl:178-196).

Workload (default): vectorised density matrix of the driven waveguide spin chain, N=40 sites,
d=4, bond dim chi=128, Lindbladian MPO of width w=8 (the exact w=6 MPO plus two zero channels),
dt=0.005, started from the all-down product state; one step = one in-place 4-stage RK4 step
(10-argument form) of the whole chain.  Metric: site-updates/s = sites x steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: device-resident state, CUDA-event timing of K steps on the library stream (max over
ranks); each rank evolves its own independent density matrix (replicas, weak scaling).
Reference arm (--impl reference): the CPU oracle (NumPy/OpenBLAS restatement of the
reference's Julia code, which cannot run here) on the host cores, rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "matrixproductstates.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOAD = dict(na=40, d=4, chi=128, w=8, dt=0.005, gam_eg=0.1, omega=0.5, gam_phi=0.1)
METRIC = "MPS site-updates/s (RK4 step, complex128)"
UNIT = "site-updates/s"
# dram__bytes_read.sum + dram__bytes_write.sum of one launch, from one ncu capture each:
# qr_kernel at the workload's interior-site QR shape (512 x 128; the input read once, the
# outputs stay in L2) and zgemm_kernel at the 3-index prod_LR shape (M=128, N=512, K=1024)
QR_TRAFFIC_BYTES = 1114624
GEMM_TRAFFIC_BYTES = 10551296


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


def oracle_step_rate(nsteps):
    """The CPU oracle (NumPy + OpenBLAS, all host threads) on the same workload."""
    from oracle import models as OM
    from oracle import mps_ref as R
    W = WORKLOAD
    na, chi, w, dt = W["na"], W["chi"], W["w"], W["dt"]
    p = OM.SpinChain(na, gam_eg=W["gam_eg"], omega=W["omega"], gam_phi=W["gam_phi"])
    rho, dims = R.mpsgroundstate(na, chi, W["d"])
    r1, r2, r3 = (R.copy_mps(rho) for _ in range(3))
    env = [R.build_env(dims, dims) for _ in range(3)]
    envop = R.build_env(dims, dims, [w] * (na + 1))
    L = [OM.construct_L_spin_model(p, 1, dt / 2, 0, w), OM.construct_L_spin_model(p, 0, 1, dt / 2, w),
         OM.construct_L_spin_model(p, 1, dt / 2, dt, w)]
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        R.RK4stp_apply_H_half_(dt, L, rho, rho, r1, r2, r3, *env, envop)
        times.append(time.perf_counter() - t0)
    return times


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


def run_reference(args, rank):
    if rank != 0:
        return None
    model, cores = cpu_info()
    W = WORKLOAD
    for _ in range(args.warmup):
        oracle_step_rate(1)
    times = oracle_step_rate(args.steps)
    tot = sum(times)
    value = W["na"] * args.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic (all-down product rho, waveguide Lindbladian)",
        "config": config_dict(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "%d full RK4 steps of the workload on the CPU oracle (NumPy/OpenBLAS %s, %d threads)"
                                   % (args.steps, model, cores)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def config_dict(args):
    W = WORKLOAD
    return {"workload": "density-matrix RK4 step, waveguide spin chain N=%d, d=%d, chi=%d, w=%d (6 + 2 zero "
                        "channels), dt=%g" % (W["na"], W["d"], W["chi"], W["w"], W["dt"]),
            "sites": W["na"], "d": W["d"], "chi": W["chi"], "w": W["w"], "dt": W["dt"],
            "parallelism": "replicas x%d (independent rho per GPU)" % args.gpus,
            "l2": "working set per step ~230 MB > 126 MB L2 (no flush needed)"}


def measure_fp64_peak(torch):
    """cuBLAS zgemm throughput (the FP64 denominator; the peaks file has HBM and bf16 only)."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    b = torch.randn(n, n, dtype=torch.complex128, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 8.0 * n ** 3 / best / 1e12


def time_gemm_mix(K, ctx, torch, stream):
    """CUDA-event timing of the zgemm kernel on the four GEMM shapes of an interior site
    (prod_LR!/update_re!/update_le! at chi=128, d=4, w=8): returns (flops, seconds) per mix."""
    import ctypes as C
    from mpsb200 import _lib
    W = WORKLOAD
    chi, d, w = W["chi"], W["d"], W["w"]
    bufs = [torch.randn(chi * w * d * chi, dtype=torch.complex128, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    p = [C.c_void_p(b.data_ptr()) for b in bufs]
    calls = [
        ("mpsb_op_prod_LR_3_4", (p[0], p[1], p[2], chi, w, chi, d, chi), 8.0 * chi * (d * chi) * (chi * w)),
        ("mpsb_op_update_re", (p[2], p[1], p[0], chi, w, d, chi, chi), 8.0 * (chi * w) * chi * (d * chi)),
        ("mpsb_op_prod_LR_4_3", (p[0], p[1], p[2], chi, d, chi, w, chi), 8.0 * (chi * d) * chi * (chi * w)),
        ("mpsb_op_update_le", (p[2], p[0], p[1], chi, d, chi, w, chi), 8.0 * (chi * w) * chi * (chi * d)),
    ]
    reps = 20
    for name, a, _ in calls:
        _lib.call(name, ctx.h, *a)
    ctx.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        for name, a, _ in calls:
            _lib.call(name, ctx.h, *a)
    e1.record(stream)
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3 / reps
    flops = sum(c[2] for c in calls)
    return flops, secs, len(calls)


def time_qr(ctx, torch, stream):
    """CUDA-event timing of one QR of the interior-site shape (d*chi x chi) through the op API:
    returns (algorithmic flops, seconds) per QR."""
    import ctypes as C
    from mpsb200 import _lib
    W = WORKLOAD
    m, n = W["d"] * W["chi"], W["chi"]
    g = torch.Generator(device="cuda").manual_seed(7)
    X = torch.randn(m * n, dtype=torch.complex128, device="cuda", generator=g)
    Q = torch.empty_like(X)
    torch.cuda.synchronize()
    args = (C.c_void_p(X.data_ptr()), C.c_void_p(Q.data_ptr()), None, m, n)
    for _ in range(3):
        _lib.call("mpsb_op_qr", ctx.h, *args)
    ctx.sync()
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        _lib.call("mpsb_op_qr", ctx.h, *args)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    return 16.0 * (m * n * n - n ** 3 / 3.0), e0.elapsed_time(e1) / 1e3 / reps, m, n


def run_serving():
    """p50/p99 job latency of a bounded sample of the mixed serving stream: 24 seeded Poisson
    arrivals at 200 jobs/s, 70% trajectories (N 20..40, chi 16/32/64, d=2, w=4) and 30%
    density matrices (N 8..16, chi 16/32, d=4, w=8), 10..30 RK4 steps each, up to 8 jobs on the
    device at once (the configuration's full sizes and 100-500 steps would run for minutes)."""
    from mpsb200 import serve as S
    jobs = S.poisson_jobs(24, 200.0, 11)
    done, st = S.Server(max_jobs=8).run(jobs)
    return {"jobs": st["jobs"], "arrival_rate_per_s": 200.0, "slots": 8,
            "latency_p50_ms": 1e3 * st["latency_p50_s"], "latency_p99_ms": 1e3 * st["latency_p99_s"],
            "queue_p50_ms": 1e3 * st["queue_p50_s"], "site_updates_per_s": st["site_updates_per_s"],
            "wall_s": st["wall_s"],
            "sample": "24 jobs: 70% trajectories N 20..40 chi<=64, 30% rho N 8..16 chi<=32, 10..30 steps"}


def run_ours(args, rank, world, local_rank, dist):
    import numpy as np
    import torch

    import mpsb200 as K
    from mpsb200 import drivers as GDR
    from mpsb200 import models as GM

    torch.cuda.set_device(local_rank)
    W = WORKLOAD
    ctx = K.Context(local_rank)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    p = GM.WaveguideChain(W["na"], gam_eg=W["gam_eg"], omega=W["omega"], gam_phi=W["gam_phi"])
    b = GDR.DensityBuffers(p, W["chi"], W["dt"], W["w"], ctx)
    dims = b.dims
    wv = [1] + [W["w"]] * (W["na"] - 1) + [1]
    fl = step_flops(dims, wv, W["d"])
    for _ in range(args.warmup):
        b.step()
    ctx.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    l0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        # one NVTX range per timed step, so a profiler can keep exactly these launches
        # (ncu --nvtx --nvtx-include "rk4_step/")
        torch.cuda.nvtx.range_push("rk4_step")
        b.step()
        torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = ctx.launches - l0
    secs = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
    value = job_rate(world, W["na"], args.steps, secs)
    tr, see, _ = b.observables(pairs=())

    # ---- end to end through the public API with host buffers: every step uploads the three
    # generator MPOs from pinned host memory (the reference loop's update_L!/update_h! refresh)
    # and reads Tr(rho) back (the measurement of the example loop)
    mpo_host = []
    h2d = 0
    for t_, (con, delt, tt) in enumerate([(1, W["dt"] / 2, 0.0), (0, 1, W["dt"] / 2), (1, W["dt"] / 2, W["dt"])]):
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
    import ctypes as C
    from mpsb200 import _lib

    def e2e_step():
        for mpo, pinned in zip(b.L, mpo_host):
            for k, (_, arr) in enumerate(pinned):
                _lib.call("mpsb_mpo_set_site", mpo.h, k + 1, arr.ctypes.data_as(C.POINTER(C.c_double)))
        b.step()
        K.scal_prod_no_conj(b.trace_fn, b.rho)

    for _ in range(args.warmup):   # the first host-buffer steps carry one-time costs
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

    # ---- roofline of the dominant kernel (the cluster QR, ~43% of the step by the ncu launch
    # list) at the workload's interior-site shape, and of the zgemm kernel on the site's GEMMs
    peak = measure_fp64_peak(torch)
    qflops, qsecs, qm, qn = time_qr(ctx, torch, stream)
    qach = qflops / qsecs / 1e12
    roofline = {"bound": "tensor", "pipe": "fp64", "limiter": "latency (128 sequential column steps)",
                "kernel": "qr_kernel (cluster Householder factorisation) + Q formation (2 zgemm_kernel, qr_tmat_kernel)",
                "achieved": qach, "peak": peak, "unit": "TFLOP/s", "frac": qach / peak,
                "peak_source": "cuBLAS zgemm 4096^3 measured in this run (no FP64 entry in MEASURED_PEAKS.json)",
                "traffic": QR_TRAFFIC_BYTES,
                "per_launch": "one QR of %d x %d (d*chi x chi): 16(mn^2 - n^3/3) = %.3e flops in %.1f us; "
                              "traffic = qr_kernel dram read+write (ncu)" % (qm, qn, qflops, qsecs * 1e6)}
    gflops, gsecs, ncalls = time_gemm_mix(K, ctx, torch, stream)
    gach = gflops / gsecs / 1e12
    roofline_gemm = {"bound": "tensor", "pipe": "fp64", "kernel": "zgemm_kernel",
                     "achieved": gach, "peak": peak, "unit": "TFLOP/s", "frac": gach / peak,
                     "traffic": GEMM_TRAFFIC_BYTES,
                     "per_launch": "flop-weighted mean over the %d GEMM shapes of an interior site "
                                   "(chi=128, d=4, w=8): %.3e flops in %.1f us; traffic = the prod_LR launch "
                                   "(M=128, N=512, K=1024) dram read+write (ncu)" % (ncalls, gflops, gsecs * 1e6)}
    serving = None
    if world == 1 and not args.no_serve:
        serving = run_serving()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic (all-down product rho, waveguide Lindbladian)",
        "config": config_dict(args),
        "clocks": clocks,
        "gpu_launches": int(launches),
        "step_tflops": sum(fl.values()) * args.steps / secs * world / 1e12,
        "step_flops": fl,
        "roofline": roofline,
        "roofline_gemm": roofline_gemm,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 16,
                "steps": ke},
        "check": {"trace_rho": tr.real, "max_see": float(np.max(see.real))},
        "serving": serving,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        model, cores = cpu_info()
        times = oracle_step_rate(1)
        line["cpu_baseline"] = {"value": W["na"] / times[0], "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": "1 full RK4 step of the workload on the CPU oracle (NumPy/OpenBLAS, "
                                          "%s, %d threads): %.2f s" % (model, cores, times[0])}
    ctx.close()
    return line


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
        bench.py --op rk4 [N] [--chi --w --slices S --random CHI0]
                                                 in-place RK4 steps of the density-matrix workload, each timed
                                                 step inside an NVTX range "rk4_step"
    """
    ap = argparse.ArgumentParser(prog="bench.py --op")
    ap.add_argument("op", choices=["qr", "gemm-mix", "zgemm", "rk4"])
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
    if a.op == "qr":
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


def main():
    if "--op" in sys.argv:
        i = sys.argv.index("--op")
        return run_op(sys.argv[i + 1:])
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream sample")
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
    line = run_ours(args, rank, world, local_rank, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
