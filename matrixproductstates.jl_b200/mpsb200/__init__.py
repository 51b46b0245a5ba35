"""mpsb200: B200-native engine for the RK4 MPS/MPO time step of jdnz/MatrixProductStates.jl.

The compute runs in libmpsb200.so (hand-written sm_100a CUDA behind the C ABI of
include/mpsb.h).  This package is the host-side mirror of the reference API.
"""
from ._lib import DimensionMismatch, MpsbError, load  # noqa: F401
from .core import (  # noqa: F401
    MPO, MPS, Arnoldi_expm_, Context, Env, RK4stp_apply_H_half_, apply_site_operator_, applyMPOtoMPS,
    build_env, compressionSVD_, compress_sum_var, compress_var_apply_H_two_site, compress_var_two_site,
    compress_sum_var_apply_H_two_site, compress_sum_var_apply_H_two_site_left, compress_sum_var_apply_H_two_site_right,
    compress_sum_var_two_site, compress_var_apply_H_two_site_left, compress_var_apply_H_two_site_right,
    RK4stp_apply_H_half_full_two_site, compress_var, compress_var_apply_H, compress_var_apply_H_left,
    compress_var_apply_H_right, compress_sum_var_apply_H, compress_sum_var_apply_H_left, compress_sum_var_apply_H_right, compress_sum_var_apply_H_, compress_sum_var_apply_H_left_,
    compress_sum_var_apply_H_right_, compress_var_apply_H_,
    compress_var_apply_H_left_, default_context, expandmps, ground_state_search_, leftorth_sites_,
    leftorthogonalizeQR_, product_mpo, steady_state_search_,
    leftorthonormalizationQR_, makemps, makempo, measure_local, mpsgroundstate, mpsproductstate,
    mpsrandom, norm_lo, normalize_lo_, scal_op_prod, scal_prod, scal_prod_no_conj,
)

__version__ = "0.1.0"
