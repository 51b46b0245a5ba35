// Small-K contraction with one local MPO tensor:
//     Out[x, m, y] = alpha * sum_k In[x, k, y] * Op[k, m] + beta * Out[x, m, y]
// with k = (k1, k2) and m = (m1, m2) split indices addressed by element strides.
//
// This is the second GEMM of prod_AOR (src/mps_base.jl:15-17) and of prod_AOL
// (src/mps_base.jl:34-37), with the reference's permutedims copies folded into the
// strides, and the site contraction of apply_site_MPOtoMPS (src/MatrixProductStates.jl:126-133).
// K = w*d and M = w*d are small (<= 64), so the whole Op tile sits in shared memory and
// each CTA streams a slab of x for one y: the kernel is bandwidth-bound and reads In / writes
// Out exactly once, coalesced along x.  A thread computes 8 outputs m of one x; the slab is 64,
// 128 or 256 wide so that every thread has outputs also when M is 8 or 16.
#include "common.cuh"

namespace mpsb {
namespace {

constexpr int NT = 256;

struct MpoParams {
  MpoApply a;
  int64_t op_k1, op_k2, op_m1, op_m2;
  bool k1_fast;  // In is contiguous along k1 (else along x)
  int tx;        // x per CTA: NT / (m-groups of 8 outputs)
};

__global__ void __launch_bounds__(NT) mpo_apply_kernel(MpoParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MpoApply& a = P.a;
  const int K = a.K1 * a.K2, M = a.M1 * a.M2;
  cd* opS = reinterpret_cast<cd*>(smem_raw);      // [k][m]  (m fastest)
  cd* inS = opS + K * M;                           // [k][x]  (x fastest)
  const int tid = threadIdx.x;
  const int TX = P.tx, G = NT / TX;
  const int x0 = blockIdx.x * TX;
  const int y = blockIdx.y;
  const int64_t bz = blockIdx.z;

  for (int e = tid; e < K * M; e += NT) {
    int m = e % M, k = e / M;
    int k1 = k % a.K1, k2 = k / a.K1, m1 = m % a.M1, m2 = m / a.M1;
    opS[e] = a.op[bz * a.op_b + k1 * P.op_k1 + k2 * P.op_k2 + m1 * P.op_m1 + m2 * P.op_m2];
  }
  const cd* in = a.in + bz * a.in_b + (int64_t)y * a.in_y;
  for (int e = tid; e < K * TX; e += NT) {
    int x, k;
    if (P.k1_fast) { k = e % K; x = e / K; }
    else           { x = e % TX; k = e / TX; }
    int k1 = k % a.K1, k2 = k / a.K1;
    int gx = x0 + x;
    inS[k * TX + x] = (gx < a.X) ? in[(int64_t)gx * a.in_x + k1 * a.in_k1 + k2 * a.in_k2] : cmk(0.0, 0.0);
  }
  __syncthreads();

  const int x = tid % TX, mg = tid / TX;   // G m-groups
  const int gx = x0 + x;
  const bool use_beta = (a.beta.x != 0.0) || (a.beta.y != 0.0);
  cd* out = a.out + bz * a.out_b + (int64_t)y * a.out_y;
  for (int mb = mg * 8; mb < M; mb += 8 * G) {
    cd acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = cmk(0.0, 0.0);
    for (int k = 0; k < K; ++k) {
      cd v = inS[k * TX + x];
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (mb + q < M) cfma(acc[q], v, opS[k * M + mb + q]);
    }
    if (gx < a.X) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        int m = mb + q;
        if (m >= M) break;
        int m1 = m % a.M1, m2 = m / a.M1;
        cd* o = out + (int64_t)gx * a.out_x + m1 * a.out_m1 + m2 * a.out_m2;
        cd v = cmul(a.alpha, acc[q]);
        if (use_beta) v = cadd(v, cmul(a.beta, *o));
        *o = v;
      }
    }
  }
}

}  // namespace

int mpo_apply_launch_strided(const MpoApply& a, int64_t op_k1, int64_t op_k2, int64_t op_m1,
                             int64_t op_m2, cudaStream_t s) {
  if (a.X <= 0 || a.Y <= 0) return MPSB_OK;
  const int K = a.K1 * a.K2, M = a.M1 * a.M2;
  if (K <= 0 || M <= 0) return MPSB_ERR_DIMENSION;
  int TX = M <= 8 ? 256 : (M <= 16 ? 128 : 64);
  while (TX > 64 && (size_t)(K * M + K * TX) * sizeof(cd) > 200 * 1024) TX /= 2;
  size_t smem = (size_t)(K * M + K * TX) * sizeof(cd);
  if (smem > 200 * 1024) return MPSB_ERR_UNSUPPORTED;
  if (a.Y > 65535 || a.batch < 1 || a.batch > 65535) return MPSB_ERR_UNSUPPORTED;
  MPSB_TRY(ensure_kernel_attrs((const void*)mpo_apply_kernel, 200 * 1024));
  MpoParams P;
  P.a = a;
  P.op_k1 = op_k1; P.op_k2 = op_k2; P.op_m1 = op_m1; P.op_m2 = op_m2;
  P.k1_fast = (a.in_k1 == 1) && (a.in_x != 1);
  P.tx = TX;
  dim3 grid((a.X + TX - 1) / TX, a.Y, a.batch);
  mpo_apply_kernel<<<grid, NT, smem, s>>>(P);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

int mpo_apply_launch(const MpoApply& a, cudaStream_t s) {
  // dense column-major Op[k, m] with ld = K
  const int K = a.K1 * a.K2;
  return mpo_apply_launch_strided(a, 1, a.K1, K, (int64_t)K * a.M1, s);
}

}  // namespace mpsb
