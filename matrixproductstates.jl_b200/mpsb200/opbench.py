"""Per-operation timing of the engine's kernels through the C-ABI (CUDA events, one GPU).

    python matrixproductstates.jl_b200/mpsb200/opbench.py qr M N [--reps R] [--warmup W]
    python matrixproductstates.jl_b200/mpsb200/opbench.py gemm-mix [--chi 128 --d 4 --w 8] [--reps R]
    python matrixproductstates.jl_b200/mpsb200/opbench.py rk4 [N] [--chi 128 --w 8] [--reps R] [--warmup W]

`qr` times mpsb_op_qr (the Householder QR of leftorth!/rightorth!, src/orthonormalisation.jl:
164-234) on a seeded random complex M x N matrix.  `gemm-mix` times the four environment
contractions of one interior site -- prod_LR (3-index L with AOR, AOL with 3-index R) and
update_re!/update_le! (src/mps_base.jl:45-262) -- at bond chi, physical d, MPO bond w.
`rk4` times in-place RK4 steps of the density-matrix workload (N sites, d=4, from the all-down
product state, dt=0.005), each timed step inside an NVTX range "rk4_step".
Prints one JSON line with microseconds per call and the algorithmic FP64 rate.  Small
enough to run under a profiler with --reps 1.
"""
import argparse
import ctypes as C
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))


def _time(torch, stream, fn, reps, warmup, ctx):
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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("op", choices=["qr", "gemm-mix", "rk4"])
    ap.add_argument("dims", nargs="*", type=int)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chi", type=int, default=128)
    ap.add_argument("--d", type=int, default=4)
    ap.add_argument("--w", type=int, default=8)
    a = ap.parse_args(argv)

    import torch
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
        us = _time(torch, stream, lambda: _lib.call("mpsb_op_qr", ctx.h, *args), a.reps, a.warmup, ctx)
        flops = 8.0 * (m * n * n - n ** 3 / 3.0) * 2   # factorisation + forming Q (complex)
        out.update({"m": m, "n": n, "us": us, "tflops": flops / us / 1e6})
    elif a.op == "rk4":
        from mpsb200 import drivers as GDR, models as GM
        na = a.dims[0] if a.dims else 40
        p = GM.WaveguideChain(na, gam_eg=0.1, omega=0.5, gam_phi=0.1)
        b = GDR.DensityBuffers(p, a.chi, 0.005, a.w, ctx)
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
        out.update({"na": na, "chi": a.chi, "w": a.w, "ms_per_step": ms, "site_updates_per_s": na / ms * 1e3})
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
            us = _time(torch, stream, lambda: _lib.call(name, ctx.h, *args), a.reps, a.warmup, ctx)
            out[tag] = {"us": us, "tflops": flops / us / 1e6}
            tot += us
        out.update({"chi": chi, "d": d, "w": w, "mix_us": tot, "mix_tflops": 4 * flops / tot / 1e6})
    ctx.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
