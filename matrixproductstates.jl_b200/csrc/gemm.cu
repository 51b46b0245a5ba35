// Complex128 strided GEMM for the environment / effective-operator contractions.
//
// Every contraction of src/mps_base.jl (prod_AOR GEMM1, prod_LR!, update_re!, update_le!,
// update_renv!, update_lenv!, ...) is a zgemm on reshaped views; here each view is an
// (m, k[, batch]) element-stride triple, so reference transposes ('), (.') and the
// reshape/permutedims chains cost no copies.
//
// Tiling (FP64 tensor path, DMMA): 64x64 complex C tile per 128-thread CTA; each warp owns
// 32x32 complex as 2x4 blocks of 16x8 and issues mma.sync.m16n8k8.f64 -- four real products
// per complex k8 step (Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br) -- with every fragment
// element loaded as one 16-byte (re, im) pair from shared memory.  K is staged 16 complex
// deep through a three-stage cp.async ring (3 x 2 x 16 x 66 x 16 B = 101 KB, two CTAs per
// SM); the row pitch of 66 elements puts the eight 16-byte fragment loads of a quarter warp
// in eight distinct bank groups.  Skinny problems split K across CTAs into a workspace that a
// second kernel sums in a fixed order, so results are bitwise reproducible run to run.
#include "common.cuh"
#include "workspace.cuh"

namespace mpsb {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 128, PAD = 2, STAGES = 3;
constexpr int LDA_S = BM + PAD, LDB_S = BN + PAD;
constexpr size_t STAGE_ELEMS = size_t(BK) * LDA_S + size_t(BK) * LDB_S;
constexpr size_t SMEM_BYTES = STAGES * STAGE_ELEMS * sizeof(cd);

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

// D (16x8, 4 per lane) += A (16x8 row, 4 per lane) * B (8x8 col, 2 per lane).  Lane l holds
// g = l/4, t = l%4: A (g, t), (g+8, t), (g, t+4), (g+8, t+4); B (t, g), (t+4, g);
// D (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1).
__device__ __forceinline__ void dmma16(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

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
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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
  const int nkt = max(0, kt1 - kt0);

  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int fg = lane >> 2, ft = lane & 3;   // fragment group / thread-in-group
  // accumulators: 2 (16-row) x 4 (8-column) blocks of the warp's 32x32 tile
  double cr[2][4][4], ci[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) cr[i][j][e] = ci[i][j][e] = 0.0;

  // prologue: STAGES-1 tiles in flight
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nkt) {
      cd* st = smem + s * STAGE_ELEMS;
      load_tile<A_MCONTIG, B_KCONTIG>(st, st + BK * LDA_S, A, B, g, m0, n0, (kt0 + s) * BK, tid);
    }
    cp_async_commit();
  }
  for (int t = 0; t < nkt; ++t) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {  // refill the stage consumed two iterations ago
      const int tn = t + STAGES - 1;
      if (tn < nkt) {
        cd* st = smem + (tn % STAGES) * STAGE_ELEMS;
        load_tile<A_MCONTIG, B_KCONTIG>(st, st + BK * LDA_S, A, B, g, m0, n0, (kt0 + tn) * BK, tid);
      }
      cp_async_commit();
    }
    const cd* As = smem + (t % STAGES) * STAGE_ELEMS;
    const cd* Bs = As + BK * LDA_S;
#pragma unroll
    for (int k8 = 0; k8 < BK; k8 += 8) {
      double ar[2][4], ai[2][4], nai[2][4], br[4][2], bi[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const cd a = As[(k8 + ft + 4 * (e >> 1)) * LDA_S + wm + 16 * i + 8 * (e & 1) + fg];
          ar[i][e] = a.x;
          ai[i][e] = CONJA ? -a.y : a.y;
          nai[i][e] = -ai[i][e];
        }
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const cd bb = Bs[(k8 + ft + 4 * e) * LDB_S + wn + 8 * j + fg];
          br[j][e] = bb.x;
          bi[j][e] = CONJB ? -bb.y : bb.y;
        }
      // Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br, term-major so one accumulator's two
      // products sit eight issues apart
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma16(cr[i][j], ar[i], br[j]);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma16(ci[i][j], ar[i], bi[j]);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma16(cr[i][j], nai[i], bi[j]);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma16(ci[i][j], ai[i], br[j]);
    }
  }
  cp_async_wait<0>();

  // accumulator (i, j, e): row wm + 16i + 8(e/2) + fg, column wn + 8j + 2ft + e%2
  if (P.splits > 1) {
    cd* W = P.ws + ((int64_t)split * g.batch + b) * (int64_t)g.M * g.N;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int m = m0 + wm + 16 * i + 8 * (e >> 1) + fg;
          const int n = n0 + wn + 8 * j + 2 * ft + (e & 1);
          if (m < g.M && n < g.N) W[(int64_t)n * g.M + m] = cmk(cr[i][j][e], ci[i][j][e]);
        }
    return;
  }
  cd* C = g.C + (int64_t)b * g.c_b;
  const bool use_beta = (g.beta.x != 0.0) || (g.beta.y != 0.0);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + 16 * i + 8 * (e >> 1) + fg;
        const int n = n0 + wn + 8 * j + 2 * ft + (e & 1);
        if (m >= g.M || n >= g.N) continue;
        cd* c = C + (int64_t)m * g.c_m + (int64_t)n * g.c_n;
        cd v = cmul(g.alpha, cmk(cr[i][j][e], ci[i][j][e]));
        if (use_beta) v = cadd(v, cmul(g.beta, *c));
        *c = v;
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
  // splits of at least two K tiles (measured on the RK4 step, 40 sites at chi=128, d=4:
  // 87.4 ms with >= 4 tiles per split from KT >= 8, 82.7 ms with >= 2 from KT >= 4)
  const int64_t basis = (ws && ws->per_problem) ? (int64_t)tiles : ctas;
  if (ws && basis < target && KT >= 4) {
    splits = (int)std::min<int64_t>((target + basis - 1) / basis, KT / 2);
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
  MPSB_TRY(ensure_kernel_attrs((const void*)fn, (int)SMEM_BYTES));
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
