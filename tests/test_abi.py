"""CPU-side checks of the drop-in boundary: the library loads and exports every symbol that
include/mpsb.h declares; the host-side model data equals the oracle's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT
from oracle import models as OM
from oracle import mps_ref as R

HEADER = os.path.join(ROOT, "include", "mpsb.h")
LIB = os.path.join(PKG_DIR, "mpsb200", "libmpsb200.so")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mpsb_[a-z0-9_A-Z]+)\s*\(", text)))


def test_header_declares_hot_path():
    syms = declared_symbols()
    for s in ("mpsb_rk4stp_apply_H_half", "mpsb_compress_sum_var_apply_H_right",
              "mpsb_compress_sum_var_apply_H_left", "mpsb_compress_var_apply_H_left", "mpsb_op_qr"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = C.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    from mpsb200 import _lib
    missing = [s for s in declared_symbols() if s not in _lib.SIGNATURES]
    assert not missing, missing


def test_ctx_create_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available() or not os.path.exists(LIB):
        pytest.skip("only meaningful on a machine without a GPU")
    import mpsb200
    with pytest.raises(mpsb200.MpsbError):
        mpsb200.Context(0)


def test_product_models_equal_oracle_models():
    from mpsb200 import models as GM
    for na in (2, 3, 7):
        po = OM.SpinChain(na, omega=0.5, gam_eg=0.1, gam_phi=0.2)
        pg = GM.WaveguideChain(na, omega=0.5, gam_eg=0.1, gam_phi=0.2)
        for (con, delt, t) in [(1, 0.005, 0.0), (0, 1, 0.3)]:
            for a, b in zip(GM.sm_hamiltonian(pg, con, delt, t), OM.sm_hamiltonian(po, con, delt, t)):
                assert a.shape == b.shape and np.array_equal(a, b)
            for w in (6, 8):
                for a, b in zip(GM.construct_L_spin_model(pg, con, delt, t, w), OM.construct_L_spin_model(po, con, delt, t, w)):
                    assert a.shape == b.shape and np.abs(a - b).max() == 0
        for a, b in zip(GM.jump_mpos(pg), OM.jump_mpos(po)):
            for x, y in zip(a, b):
                assert np.array_equal(x, y)


def test_dims_rule_host_logic():
    from mpsb200.core import _dims_rule
    for (na, dmax, d) in [(20, 32, 2), (40, 128, 4), (64, 256, 2), (3, 5, 3)]:
        assert _dims_rule(na, dmax, d) == R.dims_rule(na, dmax, d)


def test_julia_shim_binds_only_declared_symbols():
    """Every ccall of the Julia shim names an entry point that include/mpsb.h declares."""
    jl = open(os.path.join(PKG_DIR, "julia", "MatrixProductStatesB200.jl")).read()
    called = set(re.findall(r"ccall\(\(:(mpsb_[A-Za-z0-9_]+),", jl))
    assert "mpsb_rk4stp_apply_H_half" in called
    assert called <= set(declared_symbols()), sorted(called - set(declared_symbols()))
