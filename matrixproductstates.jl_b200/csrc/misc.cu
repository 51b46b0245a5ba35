// Small kernels of the sweeps: boundary-env writes, FP64 norms, rescaling, local_exp.
#include <algorithm>
#include <mutex>
#include <set>
#include <utility>

#include "common.cuh"
#include "misc.cuh"

namespace mpsb {

int ensure_kernel_attrs(const void* fn, int smem_bytes, bool cluster16) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  MPSB_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, fn})) return MPSB_OK;
  MPSB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
  if (cluster16) MPSB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  done.insert({dev, fn});
  return MPSB_OK;
}
namespace {

__global__ void set_value_kernel(cd* p, cd v) { *p = v; }

// sum |x|^2 over n complex: fixed-shape tree (deterministic), one CTA
__global__ void norm2_kernel(const cd* __restrict__ x, int64_t n, double* out) {
  __shared__ double red[1024];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s = fma(x[i].x, x[i].x, fma(x[i].y, x[i].y, s));
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// x *= 1/sqrt(*no)  (normalize_lo!: mps[end] ./ sqrt(no))
__global__ void scale_by_rsqrt_kernel(cd* x, int64_t n, const double* no) {
  const double s = sqrt(*no);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = cmk(x[i].x / s, x[i].y / s);
  }
}

// local_exp(A0, A, O) = trace(O * (A_p * A0_p')) with A_p = reshape(permutedims(A,[2,1,3]), d, :)
// (src/mps_base.jl:341-349): out = sum_{s,s'} O[s', s] sum_{a,b} A[a,s,b] conj(A0[a,s',b])
__global__ void local_exp_kernel(const cd* __restrict__ A0, const cd* __restrict__ A, const cd* __restrict__ O,
                                 int chiL, int d, int chiR, cd* out) {
  __shared__ cd red[256];
  const int npair = d * d;
  cd total = cmk(0.0, 0.0);
  for (int pair = 0; pair < npair; ++pair) {
    const int s = pair % d, s2 = pair / d;
    cd acc = cmk(0.0, 0.0);
    const int64_t nab = (int64_t)chiL * chiR;
    for (int64_t e = threadIdx.x; e < nab; e += blockDim.x) {
      int a = (int)(e % chiL);
      int64_t b = e / chiL;
      cd x = A[a + (int64_t)chiL * (s + (int64_t)d * b)];
      cd y = A0[a + (int64_t)chiL * (s2 + (int64_t)d * b)];
      cfma_cj(acc, y, x);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + w]);
      __syncthreads();
    }
    if (threadIdx.x == 0) total = cadd(total, cmul(O[s2 + d * s], red[0]));
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = total;
}

__global__ void set_value_strided_kernel(cd* p, int64_t stride, int batch, cd v) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < batch; b += gridDim.x * blockDim.x) p[b * stride] = v;
}

// one CTA per copy; the same reduction tree as norm2_kernel
__global__ void norm2_batched_kernel(const cd* __restrict__ x0, int64_t n, int64_t stride, double* out) {
  __shared__ double red[1024];
  const cd* x = x0 + (int64_t)blockIdx.x * stride;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s = fma(x[i].x, x[i].x, fma(x[i].y, x[i].y, s));
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

__global__ void scale_by_rsqrt_batched_kernel(cd* x0, int64_t n, int64_t stride, const double* no) {
  cd* x = x0 + (int64_t)blockIdx.y * stride;
  const double s = sqrt(no[blockIdx.y]);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = cmk(x[i].x / s, x[i].y / s);
}

__global__ void copy_kernel(cd* dst, const cd* src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

int grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

int set_value(cd* p, cd v, cudaStream_t s) {
  set_value_kernel<<<1, 1, 0, s>>>(p, v);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int set_value_strided(cd* p, int64_t stride, int batch, cd v, cudaStream_t s) {
  set_value_strided_kernel<<<(batch + 255) / 256, 256, 0, s>>>(p, stride, batch, v);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int norm2_batched(const cd* x, int64_t n, int64_t stride, int batch, double* out, cudaStream_t s) {
  if (batch < 1 || batch > 65535) return MPSB_ERR_UNSUPPORTED;
  norm2_batched_kernel<<<batch, 1024, 0, s>>>(x, n, stride, out);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int scale_by_rsqrt_batched(cd* x, int64_t n, int64_t stride, int batch, const double* no, cudaStream_t s) {
  if (batch < 1 || batch > 65535) return MPSB_ERR_UNSUPPORTED;
  const int gx = (int)std::min<int64_t>((n + 255) / 256, 64);
  scale_by_rsqrt_batched_kernel<<<dim3(gx, batch), 256, 0, s>>>(x, n, stride, no);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int norm2(const cd* x, int64_t n, double* out, cudaStream_t s) {
  norm2_kernel<<<1, 1024, 0, s>>>(x, n, out);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int scale_by_rsqrt(cd* x, int64_t n, const double* no, cudaStream_t s) {
  scale_by_rsqrt_kernel<<<grid_for(n), 256, 0, s>>>(x, n, no);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int local_exp(const cd* A0, const cd* A, const cd* O, int chiL, int d, int chiR, cd* out, cudaStream_t s) {
  local_exp_kernel<<<1, 256, 0, s>>>(A0, A, O, chiL, d, chiR, out);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int copy(cd* dst, const cd* src, int64_t n, cudaStream_t s) {
  if (n <= 0) return MPSB_OK;
  copy_kernel<<<grid_for(n), 256, 0, s>>>(dst, src, n);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

}  // namespace mpsb
