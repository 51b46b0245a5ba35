"""The allocation-free prod_AOR entry point (mpsb_op_prod_AOR_noalloc), through the C ABI.

It serves callers that cannot let the library call cudaMalloc (device memory owned by
their own pool allocator, or no cudaMalloc/cudaFree allowed inside their time loop); its
scratch is a fixed array inside the library.  Checked against the regular, allocating
mpsb_op_prod_AOR on two calls in a row (the second smaller, so stale contents of the shared
scratch from the first call would show), plus the size limit.  The file name sorts last so a
run that stops at the first failure has run every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import crand, empty_dev, from_dev, relerr, to_dev
from oracle import mps_ref as R

pytestmark = pytest.mark.gpu
TOL = 1e-12   # the op-level tolerance of the other kernel parity tests


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_prod_AOR_noalloc_matches_allocating_entry_point():
    import torch

    import mpsb200
    from mpsb200 import _lib

    ctx = mpsb200.Context(0)
    try:
        stream = torch.cuda.current_stream()
        for shape in [(128, 4, 128, 8, 8, 128), (17, 3, 29, 5, 3, 23)]:
            chiL, d, chiR, wL, wR, chiR0 = shape
            rng = np.random.default_rng(sum(shape))
            A, O, Rr = crand(rng, chiL, d, chiR), crand(rng, wL, d, wR, d), crand(rng, chiR, wR, chiR0)
            ref = R.prod_AOR(A, O, Rr)
            dA, dO, dR = to_dev(A), to_dev(O), to_dev(Rr)
            d_alloc, d_noalloc = empty_dev(ref.shape), empty_dev(ref.shape)
            torch.cuda.synchronize()
            _lib.call("mpsb_op_prod_AOR", ctx.h, _p(dA), _p(dO), _p(dR), _p(d_alloc), chiL, d, chiR, wL, wR, chiR0)
            ctx.sync()
            _lib.call("mpsb_op_prod_AOR_noalloc", C.c_void_p(stream.cuda_stream), _p(dA), _p(dO), _p(dR),
                      _p(d_noalloc), chiL, d, chiR, wL, wR, chiR0)
            torch.cuda.synchronize()
            got, want = from_dev(d_noalloc, ref.shape), from_dev(d_alloc, ref.shape)
            assert relerr(got, want) < TOL
            assert relerr(got, ref) < TOL
    finally:
        ctx.close()


def test_prod_AOR_noalloc_rejects_oversize():
    import torch

    from mpsb200 import _lib

    # chiL*d*wR*chiR0 = 256*4*8*256 = 2 Mi elements > the 1 Mi-element scratch: rejected on the
    # host before any launch, so the (unused) buffers can be tiny
    tiny = torch.zeros(4, dtype=torch.complex128, device="cuda")
    with pytest.raises(_lib.MpsbError) as e:
        _lib.call("mpsb_op_prod_AOR_noalloc", C.c_void_p(torch.cuda.current_stream().cuda_stream),
                  _p(tiny), _p(tiny), _p(tiny), _p(tiny), 256, 4, 256, 8, 8, 256)
    assert e.value.status == -5
    assert "16 MiB" in str(e.value)
