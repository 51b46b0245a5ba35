// Shared definitions for the mpsb200 CUDA library (sm_100a, complex128 FP64 path).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/mpsb.h"

namespace mpsb {

typedef double2 cd;  // complex128, interleaved (re, im): the Julia Complex{Float64} layout

__host__ __device__ __forceinline__ cd cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cd cadd(cd a, cd b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cd csub(cd a, cd b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cd cmul(cd a, cd b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cd cconj(cd a) { return cmk(a.x, -a.y); }
__host__ __device__ __forceinline__ cd cscale(cd a, double s) { return cmk(a.x * s, a.y * s); }
// acc += a * b
__device__ __forceinline__ void cfma(cd& acc, cd a, cd b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfma_cj(cd& acc, cd a, cd b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
// 1 / z (complex reciprocal, scaled like Smith's algorithm to avoid overflow)
__host__ __device__ __forceinline__ cd crecip(cd z) {
  double ar = fabs(z.x), ai = fabs(z.y);
  if (ar >= ai) {
    double r = z.y / z.x, den = z.x + z.y * r;
    return cmk(1.0 / den, -r / den);
  } else {
    double r = z.x / z.y, den = z.x * r + z.y;
    return cmk(r / den, -1.0 / den);
  }
}

// Error plumbing: every launch wrapper returns an mpsb status.
#define MPSB_CUDA_TRY(expr)                                   \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) {                                  \
      ::mpsb::set_last_error(_e, #expr, __FILE__, __LINE__); \
      return MPSB_ERR_CUDA;                                   \
    }                                                         \
  } while (0)

#define MPSB_TRY(expr)              \
  do {                              \
    int _s = (expr);                \
    if (_s != MPSB_OK) return _s;   \
  } while (0)

void set_last_error(cudaError_t e, const char* what, const char* file, int line);
void set_last_message(const char* fmt, ...);

// Kernel attributes are per device: set the dynamic shared-memory limit of kernel `fn` (and,
// when `cluster16`, permission for non-portable cluster sizes) once per (kernel, current device)
// in this process; thread-safe.
int ensure_kernel_attrs(const void* fn, int smem_bytes, bool cluster16 = false);

// ---------------------------------------------------------------------------------
// Strided complex GEMM descriptor: C[m,n] = alpha * sum_k opA[m,k] opB[k,n] + beta * C[m,n]
// for b in [0, batch).  Every operand is addressed by element strides, so transposes and
// the reshape/permutedims views of the reference become plain strides.
struct Gemm {
  int M = 0, N = 0, K = 0, batch = 1;
  const cd* A = nullptr; int64_t a_m = 0, a_k = 0, a_b = 0; bool conjA = false;
  const cd* B = nullptr; int64_t b_k = 0, b_n = 0, b_b = 0; bool conjB = false;
  cd* C = nullptr;       int64_t c_m = 0, c_n = 0, c_b = 0;
  cd alpha = {1.0, 0.0}, beta = {0.0, 0.0};
};

struct Workspace;  // device scratch owned by a context (engine.cu)

int gemm_launch(const Gemm& g, Workspace* ws, cudaStream_t s);

// Small-K "apply a local MPO tensor" contraction:
//   Out[x, m, y] = sum_k In[x, k, y] * Op[k, m]   with k = (k1, k2), m = (m1, m2) split indices.
struct MpoApply {
  int batch = 1;                  // problems, operands offset by the *_b strides
  int64_t in_b = 0, op_b = 0, out_b = 0;
  int X = 0, Y = 0;               // free extents
  int K1 = 0, K2 = 0, M1 = 0, M2 = 0;
  const cd* in = nullptr;  int64_t in_x = 0, in_k1 = 0, in_k2 = 0, in_y = 0;
  const cd* op = nullptr;  // dense Op[k, m], k = k1 + K1*k2, m = m1 + M1*m2, column-major (ld = K1*K2)
  cd* out = nullptr;       int64_t out_x = 0, out_m1 = 0, out_m2 = 0, out_y = 0;
  cd alpha = {1.0, 0.0}, beta = {0.0, 0.0};
};
int mpo_apply_launch(const MpoApply& a, cudaStream_t s);

// Householder QR (LAPACK zgeqrf + zungqr conventions), Q only or Q and R.
struct QrProblem {
  int m = 0, n = 0, batch = 1;
  const cd* X = nullptr; int64_t x_r = 0, x_c = 0, x_b = 0;   // input element strides (row, col, batch)
  cd* Q = nullptr;       int64_t q_r = 0, q_c = 0, q_b = 0;   // output (may alias X with equal strides)
  cd* R = nullptr;       int64_t r_r = 0, r_c = 0, r_b = 0;   // optional n x n upper-triangular factor
  int* err = nullptr;    // device word; a bounded wait that runs out sets bit 0 (may be null)
};
struct Workspace;
// Q (and R) of each problem; uses the workspace's QR scratch (V, tau, V^H V, T V1^H)
int qr_launch(const QrProblem& p, Workspace* ws, cudaStream_t s);
bool qr_supported(int m, int n);
// true when one cluster factorises an m x n problem (batched problems run in one launch)
bool qr_batch_supported(int m, int n);
// thin SVD X = U diag(S) V^H by one-sided Jacobi (S on the host, descending)
int svd_launch(int m, int n, const cd* X, int64_t x_r, int64_t x_c, cd* U, int64_t u_r, int64_t u_c, double* S,
               cd* V, int64_t v_r, int64_t v_c, Workspace* ws, cudaStream_t st);

}  // namespace mpsb
