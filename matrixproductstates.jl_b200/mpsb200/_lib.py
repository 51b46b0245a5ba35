"""ctypes binding of libmpsb200.so (include/mpsb.h).  There is no fallback: if the library
is missing or no sm_100 device is present, every entry point fails loudly."""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmpsb200.so")

OK = 0
ERRORS = {
    -1: "MPSB_ERR_INVALID_ARG", -2: "MPSB_ERR_DIMENSION", -3: "MPSB_ERR_CUDA",
    -4: "MPSB_ERR_OUT_OF_MEMORY", -5: "MPSB_ERR_UNSUPPORTED", -6: "MPSB_ERR_NONFINITE",
    -7: "MPSB_ERR_NO_DEVICE",
}


class MpsbError(RuntimeError):
    def __init__(self, status, func, msg):
        self.status = status
        super().__init__("%s returned %s: %s" % (func, ERRORS.get(status, status), msg))


class DimensionMismatch(MpsbError):
    """Shape error (the reference throws Julia's DimensionMismatch here)."""


_vp, _i, _i64, _d = C.c_void_p, C.c_int, C.c_int64, C.c_double
_pi64, _pd, _pvp = C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_void_p)

SIGNATURES = {
    "mpsb_last_error": ([], C.c_char_p),
    "mpsb_version": ([], _i),
    "mpsb_ctx_create": ([_i, _pvp], _i),
    "mpsb_ctx_destroy": ([_vp], _i),
    "mpsb_sync": ([_vp], _i),
    "mpsb_ctx_set_stream": ([_vp, _vp], _i),
    "mpsb_ctx_set_graphs": ([_vp, _i], _i),
    "mpsb_ctx_set_pipeline": ([_vp, _i], _i),
    "mpsb_ctx_set_precision": ([_vp, _i, _i], _i),
    "mpsb_ctx_set_batched_split_threshold": ([_vp, _d], _i),
    "mpsb_wait_selftest": ([_vp, _d], _i),
    "mpsb_ctx_set_profiling": ([_vp, _i], _i),
    "mpsb_ctx_profile_read": ([_vp, _pd, _pi64, _pd], _i),
    "mpsb_ctx_launch_count": ([_vp, _pi64], _i),
    "mpsb_mps_create": ([_vp, _i, _i, _pi64, _pvp], _i),
    "mpsb_mps_destroy": ([_vp], _i),
    "mpsb_mps_info": ([_vp, C.POINTER(_i), C.POINTER(_i), _pi64], _i),
    "mpsb_mps_set_site": ([_vp, _i, _pd], _i),
    "mpsb_mps_get_site": ([_vp, _i, _pd], _i),
    "mpsb_mps_site_ptr": ([_vp, _i, _pvp], _i),
    "mpsb_mps_copy": ([_vp, _vp], _i),
    "mpsb_mps_create_batch": ([_vp, _i, _i, _pi64, _i, _pvp], _i),
    "mpsb_env_create_batch": ([_vp, _i, _pi64, _pi64, _pi64, _i, _pvp], _i),
    "mpsb_mps_batch": ([_vp, C.POINTER(_i)], _i),
    "mpsb_mps_set_site_copy": ([_vp, _i, _i, _pd], _i),
    "mpsb_mps_get_site_copy": ([_vp, _i, _i, _pd], _i),
    "mpsb_mps_view": ([_vp, _i, _pvp], _i),
    "mpsb_mps_select": ([_vp, _pvp, _i, C.POINTER(_i)], _i),
    "mpsb_normalize_lo_batch": ([_vp, _vp, _pd], _i),
    "mpsb_mpo_create": ([_vp, _i, _i, _pi64, _pvp], _i),
    "mpsb_mpo_destroy": ([_vp], _i),
    "mpsb_mpo_set_site": ([_vp, _i, _pd], _i),
    "mpsb_mpo_get_site": ([_vp, _i, _pd], _i),
    "mpsb_env_create": ([_vp, _i, _pi64, _pi64, _pi64, _pvp], _i),
    "mpsb_env_destroy": ([_vp], _i),
    "mpsb_env_get": ([_vp, _i, _pd], _i),
    "mpsb_env_set": ([_vp, _i, _pd], _i),
    "mpsb_rk4stp_apply_H_half": ([_vp, _d] + [_vp] * 12, _i),
    "mpsb_compress_var_apply_H_left": ([_vp] * 6, _i),
    "mpsb_compress_sum_var_apply_H_right": ([_vp, _vp, _pvp, _vp, _vp, _pd, _i, _pvp, _vp], _i),
    "mpsb_compress_sum_var_apply_H_left": ([_vp, _vp, _pvp, _vp, _vp, _pd, _i, _pvp, _vp], _i),
    "mpsb_compress_var_apply_H": ([_vp] * 6 + [_i], _i),
    "mpsb_compress_sum_var_apply_H": ([_vp, _vp, _vp, _pd, _i, _pvp, _vp, _i], _i),
    "mpsb_compress_sum_var": ([_vp, _vp, _vp, _pd, _i, _pvp, _i], _i),
    "mpsb_ground_state_search": ([_vp, _vp, _vp, _i, _d, _d, _pd], _i),
    "mpsb_normalize_lo": ([_vp, _vp, _pd], _i),
    "mpsb_norm_lo": ([_vp, _vp, _pd], _i),
    "mpsb_leftorthonormalizationQR": ([_vp, _vp, _pd], _i),
    "mpsb_leftorthogonalizeQR": ([_vp, _vp, _pd], _i),
    "mpsb_apply_site_operator": ([_vp, _vp, _i, _pd], _i),
    "mpsb_scal_prod": ([_vp, _vp, _vp, _pd], _i),
    "mpsb_scal_op_prod": ([_vp, _vp, _vp, _vp, _pd], _i),
    "mpsb_scal_prod_no_conj": ([_vp, _vp, _vp, _pd], _i),
    "mpsb_measure_local": ([_vp, _vp, _pd, _pd], _i),
    "mpsb_apply_mpo_to_mps": ([_vp, _vp, _vp, _vp], _i),
    "mpsb_op_prod_AOR": ([_vp] * 5 + [_i] * 6, _i),
    "mpsb_op_prod_AOL": ([_vp] * 5 + [_i] * 6, _i),
    "mpsb_op_prod_LR_3_4": ([_vp] * 4 + [_i] * 5, _i),
    "mpsb_op_prod_LR_4_3": ([_vp] * 4 + [_i] * 5, _i),
    "mpsb_op_update_re": ([_vp] * 4 + [_i] * 5, _i),
    "mpsb_op_update_le": ([_vp] * 4 + [_i] * 5, _i),
    "mpsb_compression_svd": ([_vp, _vp, _i, _d, _pvp, _pd, _pd, _pd], _i),
    "mpsb_compress_var_apply_H_two_site": ([_vp, _vp, _vp, _vp, _i, _d, _i, _pvp], _i),
    "mpsb_compress_sum_var_apply_H_two_site": ([_vp, _vp, _pd, _i, _pvp, _vp, _i, _d, _i, _i, _pvp], _i),
    "mpsb_op_svd": ([_vp, _vp, _vp, _pd, _vp, _i, _i], _i),
    "mpsb_op_qr": ([_vp] * 4 + [_i] * 2, _i),
    "mpsb_op_zgemm": ([_vp, _i, _i, _i, _vp, _i64, _i64, _i, _vp, _i64, _i64, _i, _vp, _i64, _i64, _pd, _pd, _i], _i),
    "mpsb_op_prod_AOR_noalloc": ([_vp] * 5 + [_i] * 6, _i),
}

_lib = None


def load():
    """Load the in-tree library (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libmpsb200.so not built at %s (run matrixproductstates.jl_b200/build.py)" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def call(name, *args):
    lib = load()
    st = getattr(lib, name)(*args)
    if st != OK:
        msg = lib.mpsb_last_error().decode(errors="replace")
        cls = DimensionMismatch if st == -2 else MpsbError
        raise cls(st, name, msg)
    return st
