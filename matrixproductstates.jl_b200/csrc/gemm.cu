// Complex128 strided GEMM for the environment / effective-operator contractions.
//
// Every contraction of src/mps_base.jl (prod_AOR GEMM1, prod_LR!, update_re!, update_le!,
// update_renv!, update_lenv!, ...) is a zgemm on reshaped views; here each view is an
// (m, k[, batch]) element-stride triple, so reference transposes ('), (.') and the
// reshape/permutedims chains cost no copies.
//
// Tiling (FP64 pipe, DFMA): 64x64 complex C tile per 256-thread CTA, each thread owns a
// 4x4 complex micro-tile strided by 16 (so A fragments are read as 16 consecutive complex,
// B fragments are warp broadcasts), K staged 16 complex deep through a two-stage cp.async
// ring in dynamic shared memory (2 x 2 x 16 x 65 x 16 B = 66.5 KB).  Skinny problems split
// K across CTAs into a workspace that a second kernel sums in a fixed order, so results
// are bitwise reproducible run to run.
#include "common.cuh"
#include "workspace.cuh"

namespace mpsb {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256, PAD = 1;
constexpr int LDA_S = BM + PAD, LDB_S = BN + PAD;
constexpr size_t STAGE_ELEMS = size_t(BK) * LDA_S + size_t(BK) * LDB_S;
constexpr size_t SMEM_BYTES = 2 * STAGE_ELEMS * sizeof(cd);

struct GemmParams {
  Gemm g;
  int splits;
  int kt_per_split;   // K tiles per split
  cd* ws;             // [split][batch][N][M] partials when splits > 1
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <bool A_MCONTIG, bool B_KCONTIG>
__device__ __forceinline__ void load_tile(cd* As, cd* Bs, const cd* A, const cd* B, const Gemm& g,
                                          int m0, int n0, int k0, int tid) {
  // A tile: BM x BK, stored As[k][m]
#pragma unroll
  for (int i = 0; i < (BM * BK) / NT; ++i) {
    int m, k;
    if (A_MCONTIG) { m = tid % BM; k = tid / BM + (NT / BM) * i; }
    else           { k = tid % BK; m = tid / BK + (NT / BK) * i; }
    int gm = m0 + m, gk = k0 + k;
    bool ok = (gm < g.M) && (gk < g.K);
    const cd* src = ok ? (A + (int64_t)gm * g.a_m + (int64_t)gk * g.a_k) : A;
    cp_async16(As + k * LDA_S + m, src, ok);
  }
  // B tile: BK x BN, stored Bs[k][n]
#pragma unroll
  for (int i = 0; i < (BN * BK) / NT; ++i) {
    int n, k;
    if (B_KCONTIG) { k = tid % BK; n = tid / BK + (NT / BK) * i; }
    else           { n = tid % BN; k = tid / BN + (NT / BN) * i; }
    int gn = n0 + n, gk = k0 + k;
    bool ok = (gn < g.N) && (gk < g.K);
    const cd* src = ok ? (B + (int64_t)gk * g.b_k + (int64_t)gn * g.b_n) : B;
    cp_async16(Bs + k * LDB_S + n, src, ok);
  }
}

template <bool CONJA, bool CONJB, bool A_MCONTIG, bool B_KCONTIG>
__global__ void __launch_bounds__(NT, 2) zgemm_kernel(GemmParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* smem = reinterpret_cast<cd*>(smem_raw);
  const Gemm& g = P.g;
  const int tid = threadIdx.x;
  const int tiles_m = (g.M + BM - 1) / BM;
  const int m0 = (blockIdx.x % tiles_m) * BM;
  const int n0 = (blockIdx.x / tiles_m) * BN;
  const int split = blockIdx.y;
  const int b = blockIdx.z;
  const cd* A = g.A + (int64_t)b * g.a_b;
  const cd* B = g.B + (int64_t)b * g.b_b;

  const int KT = (g.K + BK - 1) / BK;
  const int kt0 = split * P.kt_per_split;
  const int kt1 = min(KT, kt0 + P.kt_per_split);

  const int tm = tid % 16, tn = tid / 16;
  cd acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = cmk(0.0, 0.0);

  if (kt0 < kt1) {
    load_tile<A_MCONTIG, B_KCONTIG>(smem, smem + BK * LDA_S, A, B, g, m0, n0, kt0 * BK, tid);
    cp_async_commit();
    for (int kt = kt0; kt < kt1; ++kt) {
      const int st = (kt - kt0) & 1;
      if (kt + 1 < kt1) {
        cd* nxt = smem + (st ^ 1) * STAGE_ELEMS;
        load_tile<A_MCONTIG, B_KCONTIG>(nxt, nxt + BK * LDA_S, A, B, g, m0, n0, (kt + 1) * BK, tid);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      const cd* As = smem + st * STAGE_ELEMS;
      const cd* Bs = As + BK * LDA_S;
#pragma unroll 4
      for (int k = 0; k < BK; ++k) {
        cd a[4], bb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          a[i] = As[k * LDA_S + tm + 16 * i];
          if (CONJA) a[i].y = -a[i].y;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          bb[j] = Bs[k * LDB_S + tn + 16 * j];
          if (CONJB) bb[j].y = -bb[j].y;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) cfma(acc[i][j], a[i], bb[j]);
      }
      __syncthreads();
    }
  }

  if (P.splits > 1) {
    cd* W = P.ws + ((int64_t)split * g.batch + b) * (int64_t)g.M * g.N;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int m = m0 + tm + 16 * i;
      if (m >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int n = n0 + tn + 16 * j;
        if (n < g.N) W[(int64_t)n * g.M + m] = acc[i][j];
      }
    }
    return;
  }
  cd* C = g.C + (int64_t)b * g.c_b;
  const bool use_beta = (g.beta.x != 0.0) || (g.beta.y != 0.0);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int m = m0 + tm + 16 * i;
    if (m >= g.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int n = n0 + tn + 16 * j;
      if (n >= g.N) continue;
      cd* c = C + (int64_t)m * g.c_m + (int64_t)n * g.c_n;
      cd v = cmul(g.alpha, acc[i][j]);
      if (use_beta) v = cadd(v, cmul(g.beta, *c));
      *c = v;
    }
  }
}

__global__ void splitk_reduce_kernel(Gemm g, int splits, const cd* __restrict__ ws) {
  const int64_t MN = (int64_t)g.M * g.N;
  const int64_t total = MN * g.batch;
  const bool use_beta = (g.beta.x != 0.0) || (g.beta.y != 0.0);
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = idx / MN, r = idx % MN;
    int m = (int)(r % g.M), n = (int)(r / g.M);
    cd s = cmk(0.0, 0.0);
    for (int q = 0; q < splits; ++q) s = cadd(s, ws[((int64_t)q * g.batch + b) * MN + r]);
    cd* c = g.C + b * g.c_b + (int64_t)m * g.c_m + (int64_t)n * g.c_n;
    cd v = cmul(g.alpha, s);
    if (use_beta) v = cadd(v, cmul(g.beta, *c));
    *c = v;
  }
}

__global__ void scale_c_kernel(Gemm g) {
  // K == 0: C = beta * C
  const int64_t MN = (int64_t)g.M * g.N, total = MN * g.batch;
  const bool use_beta = (g.beta.x != 0.0) || (g.beta.y != 0.0);
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = idx / MN, r = idx % MN;
    int m = (int)(r % g.M), n = (int)(r / g.M);
    cd* c = g.C + b * g.c_b + (int64_t)m * g.c_m + (int64_t)n * g.c_n;
    *c = use_beta ? cmul(g.beta, *c) : cmk(0.0, 0.0);
  }
}

typedef void (*KernelFn)(GemmParams);

template <bool CA, bool CB>
KernelFn pick_layout(bool amc, bool bkc) {
  if (amc) return bkc ? zgemm_kernel<CA, CB, true, true> : zgemm_kernel<CA, CB, true, false>;
  return bkc ? zgemm_kernel<CA, CB, false, true> : zgemm_kernel<CA, CB, false, false>;
}

KernelFn pick(const Gemm& g) {
  bool amc = (g.a_m == 1), bkc = (g.b_k == 1);
  if (g.conjA) return g.conjB ? pick_layout<true, true>(amc, bkc) : pick_layout<true, false>(amc, bkc);
  return g.conjB ? pick_layout<false, true>(amc, bkc) : pick_layout<false, false>(amc, bkc);
}

}  // namespace

int gemm_launch(const Gemm& g, Workspace* ws, cudaStream_t s) {
  if (g.M < 0 || g.N < 0 || g.K < 0 || g.batch < 1) return MPSB_ERR_DIMENSION;
  if (g.M == 0 || g.N == 0) return MPSB_OK;
  if (g.batch > 65535) return MPSB_ERR_UNSUPPORTED;
  count_launch(ws);
  if (g.K == 0) {
    int64_t total = (int64_t)g.M * g.N * g.batch;
    int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
    scale_c_kernel<<<blocks, 256, 0, s>>>(g);
    MPSB_CUDA_TRY(cudaGetLastError());
    return MPSB_OK;
  }
  const int tiles = ((g.M + BM - 1) / BM) * ((g.N + BN - 1) / BN);
  const int KT = (g.K + BK - 1) / BK;
  const int64_t ctas = (int64_t)tiles * g.batch;
  int splits = 1;
  const int target = 2 * 148;  // two resident 64x64 tiles per SM
  // without a workspace (ws == nullptr) K is never split, so no scratch is needed
  if (ws && ctas < target && KT >= 8) {
    splits = (int)std::min<int64_t>((target + ctas - 1) / ctas, KT / 4);
    splits = std::max(1, std::min(splits, 32));
  }
  int kt_per = (KT + splits - 1) / splits;
  splits = (KT + kt_per - 1) / kt_per;

  GemmParams P;
  P.g = g;
  P.splits = splits;
  P.kt_per_split = kt_per;
  P.ws = nullptr;
  if (splits > 1) {
    size_t bytes = (size_t)splits * g.batch * g.M * g.N * sizeof(cd);
    MPSB_TRY(ws_splitk(ws, bytes, &P.ws));
  }
  KernelFn fn = pick(g);
  static bool attr_done[16] = {false};
  int key = (g.conjA ? 8 : 0) | (g.conjB ? 4 : 0) | (g.a_m == 1 ? 2 : 0) | (g.b_k == 1 ? 1 : 0);
  if (!attr_done[key]) {
    MPSB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    attr_done[key] = true;
  }
  dim3 grid(tiles, splits, g.batch);
  fn<<<grid, NT, SMEM_BYTES, s>>>(P);
  MPSB_CUDA_TRY(cudaGetLastError());
  if (splits > 1) {
    count_launch(ws);
    int64_t total = (int64_t)g.M * g.N * g.batch;
    int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
    splitk_reduce_kernel<<<blocks, 256, 0, s>>>(g, splits, P.ws);
    MPSB_CUDA_TRY(cudaGetLastError());
  }
  return MPSB_OK;
}

}  // namespace mpsb
