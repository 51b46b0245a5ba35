#pragma once
#include "common.cuh"

namespace mpsb {
int set_value(cd* p, cd v, cudaStream_t s);
// p[b * stride] = v for b < batch
int set_value_strided(cd* p, int64_t stride, int batch, cd v, cudaStream_t s);
// out[b] = sum |x[b * stride + i]|^2 over i < n, one fixed-shape tree per copy
int norm2_batched(const cd* x, int64_t n, int64_t stride, int batch, double* out, cudaStream_t s);
// x[b * stride + i] /= sqrt(no[b])
int scale_by_rsqrt_batched(cd* x, int64_t n, int64_t stride, int batch, const double* no, cudaStream_t s);
int norm2(const cd* x, int64_t n, double* out, cudaStream_t s);
int scale_by_rsqrt(cd* x, int64_t n, const double* no, cudaStream_t s);
int local_exp(const cd* A0, const cd* A, const cd* O, int chiL, int d, int chiR, cd* out, cudaStream_t s);
int copy(cd* dst, const cd* src, int64_t n, cudaStream_t s);
int mpo_apply_launch_strided(const MpoApply& a, int64_t op_k1, int64_t op_k2, int64_t op_m1,
                             int64_t op_m2, cudaStream_t s);
}  // namespace mpsb
