// Split-precision complex GEMM on the 5th-generation tensor cores (tcgen05, kind::i8).
//
// The environment and effective-operator contractions of src/mps_base.jl (prod_AOR's first
// GEMM, prod_AOL's first GEMM, prod_LR!, update_re!, update_le!, update_renv!, update_lenv!)
// are complex128 GEMMs C = alpha op(A) op(B) + beta C.  tcgen05 has no FP64 kind, so this path
// writes each FP64 operand as a sum of S integer slices and multiplies the slices on the int8
// tensor pipe, where products accumulate exactly in int32 (the Ozaki scheme):
//
//   * complex -> real: C' (M x 2N) = A' (M x 2K) B' (2K x 2N) with A' rows the interleaved
//     (re, im) pairs of A's rows and B' column pairs (n,re) = [re, -im ...], (n,im) = [im, re ...]
//     of B's columns, so one real GEMM gives both components;
//   * each row r of A' (column of B') gets an exponent E_r with |x| < 2^E_r, and the scaled row
//     x 2^(7-E_r) is peeled into digits d_0..d_{S-1} in [-127, 127] with
//     x = 2^E_r sum_i 2^(-7(i+1)) d_i + O(2^(E_r - 7S))   (exact FP64 arithmetic);
//   * level t = i + j collects every slice product A_i B_j of the same weight 2^(-7(t+2)) in one
//     int32 TMEM accumulator (exact: |sum| <= S * 127^2 * 2K < 2^31 for 2K < 2^17 / S);
//     levels t < S are kept (S(S+1)/2 MMAs per k-step), the rest are the truncation;
//   * the epilogue reads the S accumulators, sums them in FP64 from the smallest weight up,
//     applies 2^(E_a + E_b), alpha and beta, and writes complex128 C through its strides.
//
// Kernel (persistent: one CTA per SM, 384 threads, 128 x 64 tiles of C' of every problem taken
// round-robin): warp 0 issues TMA loads of the 2S slice tiles of each 64-byte k-stage (64B
// swizzle) into a shared-memory ring that runs on across tiles; warp 1 owns the TMEM allocation
// and one lane issues tcgen05.mma for all slice pairs of a stage -- row i of the slice triangle,
// A_i [B_0 .. B_{S-1-i}], as MMAs of N up to 256 whose output columns are the consecutive level
// accumulators -- and commits the stage back to the producer; warps 4..11 are the epilogue (two
// warps per TMEM lane quarter, one 32-column half each), which hands the accumulators back as
// soon as it has read them, so the next tile's loads and MMAs overlap its FP64 combination and
// stores.  Every wait is bounded in wall-clock time: a wait that runs out sets the context's
// error word and the CTA winds down (copies in flight land, no MMA is left running, the TMEM
// allocation is released).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "ozaki.cuh"
#include "workspace.cuh"

namespace mpsb {

namespace {

constexpr int OZ_BM = 128;        // rows of A' per tile (tcgen05 M)
constexpr int OZ_BN = 64;         // columns of C' per tile (tcgen05 N): 32 complex columns
constexpr int OZ_BK = 64;         // int8 k per stage: one 64-byte swizzled row
constexpr int OZ_KP_ALIGN = 64;   // K' padding
constexpr int A_TILE = OZ_BM * OZ_BK;   // 8 KB
constexpr int B_TILE = OZ_BN * OZ_BK;   // 4 KB
constexpr int OZ_THREADS = 384;   // warp 0 TMA, warp 1 TMEM + MMA, warps 2-3 idle, warps 4-11 epilogue
constexpr int OZ_EPI_WARPS = 8;
constexpr unsigned long long WAIT_NS = 2000000000ull;   // a bounded mbarrier wait gives up after 2 s

__host__ __device__ constexpr int stage_bytes(int S) { return S * (A_TILE + B_TILE); }
__host__ __device__ constexpr int num_stages(int S) {
  return (220 * 1024) / stage_bytes(S) > 4 ? 4 : (220 * 1024) / stage_bytes(S);
}
__host__ __device__ constexpr int tmem_cols(int S) { return S * OZ_BN <= 256 ? 256 : 512; }
__host__ __device__ constexpr int smem_bytes(int S) { return 1024 + num_stages(S) * stage_bytes(S) + 256; }

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// non-blocking test of the phase of the given parity
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// wait for the phase of the given parity, bounded in wall-clock time; false when it ran out
__device__ __noinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns = WAIT_NS) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned i = 1;; ++i) {
    if (mbar_test(bar, parity)) return true;
    if ((i & 255) == 0 && global_ns() - t0 > limit_ns) return false;
    __nanosleep(32);
  }
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
// K-major operand with 64-byte swizzle: rows of 64 bytes, 8-row groups 512 bytes apart
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);        // start address
  d |= (uint64_t)1 << 16;                        // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;               // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                        // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                        // layout: 64-byte swizzle
  return d;
}
// instruction descriptor: kind::i8, signed A and B, s32 accumulator, both K-major, M=128, N=n
// (a multiple of 16 up to 256)
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);
}
// B slices one MMA covers: N = OZ_BN per slice, at most 256
constexpr int OZ_SLICES_PER_MMA = 256 / OZ_BN;
// A-operand collector use across consecutive MMAs that share A: 0 = read A (no reuse),
// 1 = read and keep it, 2 = reuse the kept A, 3 = reuse it for the last time
#define MPSB_MMA_I8(QUAL)                                                                          \
  asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"                                        \
               "tcgen05.mma.cta_group::1.kind::i8" QUAL " [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d), \
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)                                  \
               : "memory")
template <int COLLECT>
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  if (COLLECT == 1) MPSB_MMA_I8(".collector::a::fill");
  else if (COLLECT == 2) MPSB_MMA_I8(".collector::a::use");
  else if (COLLECT == 3) MPSB_MMA_I8(".collector::a::lastuse");
  else MPSB_MMA_I8("");
}
#undef MPSB_MMA_I8
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// ---------------------------------------------------------------- slicing
// A view of the operand whose rows become rows of the sliced matrix: element (r, k) at
// X[r * x_r + k * x_k], conjugated when conj.  In B mode a row (a column n of op(B)) becomes
// the pair of rows (n,re) = [re, -im], (n,im) = [im, re] of B'^T; otherwise a row is [re, im].
struct SliceView {
  const cd* X; int R, K; int64_t x_r, x_k; bool conj;
  int64_t x_bat;   // element offset between the problems of a batch (blockIdx.z)
};

// biased IEEE exponent of max(|re|, |im|) (0 for zero / subnormal), max-reduced per row into
// rexp (zeroed before).  A CTA covers 32 rows and kper tiles of 32 columns, keeping a running
// maximum per thread: for large operands several loads per thread are in flight and one atomic
// per row and CTA remains, small ones keep one tile per CTA and the grid wide.
__global__ void oz_rowexp_kernel(SliceView v, int* __restrict__ rexp0, int64_t rexp_bat, int kper) {
  __shared__ int tile_e[32][33];
  const int r0 = blockIdx.x * 32;
  v.X += (int64_t)blockIdx.z * v.x_bat;
  int* rexp = rexp0 + (int64_t)blockIdx.z * rexp_bat;
  const int tid = threadIdx.x;
  const bool rc = (v.x_r == 1);   // rows contiguous: lanes run along r
  const int kt0 = blockIdx.y * kper, kt1 = min((v.K + 31) / 32, kt0 + kper);
  int em[4] = {0, 0, 0, 0};
#pragma unroll 2
  for (int kt = kt0; kt < kt1; ++kt) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int rr, kk;
      if (rc) { rr = tid % 32; kk = tid / 32 + 8 * i; }
      else    { kk = tid % 32; rr = tid / 32 + 8 * i; }
      const int r = r0 + rr, k = kt * 32 + kk;
      if (r < v.R && k < v.K) {
        const cd x = v.X[(int64_t)r * v.x_r + (int64_t)k * v.x_k];
        const double m = fmax(fabs(x.x), fabs(x.y));
        em[i] = max(em[i], (int)((__double_as_longlong(m) >> 52) & 0x7FF));
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (rc) tile_e[tid % 32][tid / 32 + 8 * i] = em[i];
    else    tile_e[tid / 32 + 8 * i][tid % 32] = em[i];
  }
  __syncthreads();
  const int warp = tid / 32, lane = tid % 32;
  for (int rr = warp; rr < 32; rr += 8) {
    int e = tile_e[rr][lane];
    for (int o = 16; o; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
    if (lane == 0 && e > 0 && r0 + rr < v.R) atomicMax(rexp + r0 + rr, e);
  }
}

// 2^k for -1022 <= k <= 1023, written into the exponent field
__device__ __forceinline__ double pow2_exact(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// The scaling x -> x 2^(7-e) of a row whose maximum has the biased exponent E (e = E - 1022, its
// frexp exponent) as two exact multiplications x * s1 * s2 (2^(7-e) itself overflows for E < 6);
// a row of zeros and subnormals (E = 0) gets s2 = 0.
struct RowScale {
  double s1, s2;
};
__device__ __forceinline__ RowScale row_scale(int E) {
  const int k = 1029 - E;
  RowScale r;
  r.s1 = (k > 1023) ? pow2_exact(512) : 1.0;
  r.s2 = (E > 0) ? pow2_exact(k > 1023 ? k - 512 : k) : 0.0;
  return r;
}

// Balanced base-128 digits of x 2^(7-e) in (-128, 128): d_i = round-to-nearest-even of the
// remainder clamped to [-127, 127], every step exact in FP64.  The clamp matters at every digit:
// x just below a power of two (1 - 1e-12, say) gives a run of remainders in (127, 128).
template <int S>
__device__ __forceinline__ void digits(double x, RowScale rs, int (&d)[S]) {
  double t = (x * rs.s1) * rs.s2;
#pragma unroll
  for (int i = 0; i < S; ++i) {
    const int q = max(-127, min(127, __double2int_rn(t)));
    d[i] = q;
    if (i + 1 < S) t = (t - (double)q) * 128.0;
  }
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  // the low bytes of a, b, c, d (their int8 values) as bytes 0..3
  return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// The S digit slices of 4 consecutive complex k of row r, at byte kbyte of each slice row (8
// bytes): A mode writes row r as [re, im] pairs; B mode writes the row pair 2r (n,re) = [re, -im]
// and 2r+1 (n,im) = [im, re].
template <int S, bool BMODE>
__device__ __forceinline__ void store_digits(int8_t* __restrict__ out, int64_t rows_out, int Kp, int r, int64_t kbyte,
                                             const cd (&x)[4], RowScale rs) {
  int dre[4][S], dim[4][S];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    digits<S>(x[j].x, rs, dre[j]);
    digits<S>(x[j].y, rs, dim[j]);
  }
#pragma unroll
  for (int t = 0; t < S; ++t) {
    if (!BMODE) {
      int8_t* p = out + ((int64_t)t * rows_out + r) * Kp + kbyte;
      *reinterpret_cast<uint2*>(p) = make_uint2(pack4(dre[0][t], dim[0][t], dre[1][t], dim[1][t]),
                                                pack4(dre[2][t], dim[2][t], dre[3][t], dim[3][t]));
    } else {
      int8_t* p = out + ((int64_t)t * rows_out + 2 * (int64_t)r) * Kp + kbyte;
      *reinterpret_cast<uint2*>(p) = make_uint2(pack4(dre[0][t], -dim[0][t], dre[1][t], -dim[1][t]),
                                                pack4(dre[2][t], -dim[2][t], dre[3][t], -dim[3][t]));
      *reinterpret_cast<uint2*>(p + Kp) = make_uint2(pack4(dim[0][t], dre[0][t], dim[1][t], dre[1][t]),
                                                     pack4(dim[2][t], dre[2][t], dim[3][t], dre[3][t]));
    }
  }
}

// Digits of a 32-row x 32-complex tile: out[t][row][k'] (K' = 2K padded to Kp, rows padded to
// the tile grid with zeros, so every byte the GEMM reads is written).
template <int S, bool BMODE>
__global__ void oz_split_kernel(SliceView v, const int* __restrict__ rexp0, int64_t rexp_bat, int8_t* __restrict__ out0,
                                int64_t rows_out, int Kp) {
  __shared__ cd tile[32][33];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  v.X += (int64_t)blockIdx.z * v.x_bat;
  const int* rexp = rexp0 + (int64_t)blockIdx.z * rexp_bat;
  int8_t* out = out0 + (int64_t)blockIdx.z * S * rows_out * Kp;
  const int tid = threadIdx.x;
  const bool rc = (v.x_r == 1);
  for (int i = 0; i < 4; ++i) {
    int rr, kk;
    if (rc) { rr = tid % 32; kk = tid / 32 + 8 * i; }
    else    { kk = tid % 32; rr = tid / 32 + 8 * i; }
    const int r = r0 + rr, k = k0 + kk;
    cd x = cmk(0.0, 0.0);
    if (r < v.R && k < v.K) {
      x = v.X[(int64_t)r * v.x_r + (int64_t)k * v.x_k];
      if (v.conj) x.y = -x.y;
    }
    tile[rr][kk] = x;
  }
  __syncthreads();
  // thread -> (row, 4 consecutive complex k)
  const int rr = tid / 8, kq = (tid % 8) * 4;
  const int r = r0 + rr;
  const RowScale rs = row_scale((r < v.R) ? rexp[r] : 0);
  const cd xs[4] = {tile[rr][kq], tile[rr][kq + 1], tile[rr][kq + 2], tile[rr][kq + 3]};
  store_digits<S, BMODE>(out, rows_out, Kp, r, 2 * (int64_t)(k0 + kq), xs, rs);
}

// Exponent scan and slicing fused, for operands whose rows fit in shared memory: a CTA holds
// `rpc` whole rows (all Kc complex columns of the slice grid, zeros beyond K), takes each row's
// largest exponent and writes its digits -- one read of the operand instead of two and no
// atomics.  rpc divides 32, so the grid covers the padded rows exactly (rows >= R get exponent
// 0 and zero digits); exponents and digits are those of the two-pass kernels.
constexpr int OZ_FUSED_SMEM = 96 * 1024;
template <int S, bool BMODE>
__global__ void __launch_bounds__(256)
    oz_slice_rows_kernel(SliceView v, int* __restrict__ rexp0, int64_t rexp_bat, int8_t* __restrict__ out0,
                         int64_t rows_out, int Kp, int rpc) {
  extern __shared__ __align__(16) unsigned char rows_smem[];
  cd* tile = reinterpret_cast<cd*>(rows_smem);   // [rpc][Kc + 1]
  __shared__ int rowE[32];
  const int Kc = Kp / 2, ld = Kc + 1;
  const int r0 = blockIdx.x * rpc;
  v.X += (int64_t)blockIdx.z * v.x_bat;
  int* rexp = rexp0 + (int64_t)blockIdx.z * rexp_bat;
  int8_t* out = out0 + (int64_t)blockIdx.z * S * rows_out * Kp;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const bool rc = (v.x_r == 1);   // rows contiguous: consecutive threads take consecutive rows
  const int n = rpc * Kc;
  for (int e = tid; e < n; e += 256) {
    int rr, k;
    if (rc) { rr = e % rpc; k = e / rpc; }
    else    { k = e % Kc; rr = e / Kc; }
    const int r = r0 + rr;
    cd x = cmk(0.0, 0.0);
    if (r < v.R && k < v.K) {
      x = v.X[(int64_t)r * v.x_r + (int64_t)k * v.x_k];
      if (v.conj) x.y = -x.y;
    }
    tile[rr * ld + k] = x;
  }
  __syncthreads();
  for (int rr = warp; rr < rpc; rr += 8) {
    int e = 0;
    for (int k = lane; k < Kc; k += 32) {
      const cd x = tile[rr * ld + k];
      e = max(e, (int)((__double_as_longlong(fmax(fabs(x.x), fabs(x.y))) >> 52) & 0x7FF));
    }
    for (int o = 16; o; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
    if (lane == 0) {
      rowE[rr] = e;
      if (r0 + rr < v.R) rexp[r0 + rr] = e;
    }
  }
  __syncthreads();
  const int q4 = Kc / 4;   // items of 4 complex k per row
  for (int it = tid; it < rpc * q4; it += 256) {
    const int rr = it / q4, kq = (it % q4) * 4;
    const int r = r0 + rr;
    const cd* tp = tile + rr * ld + kq;
    const cd xs[4] = {tp[0], tp[1], tp[2], tp[3]};
    store_digits<S, BMODE>(out, rows_out, Kp, r, 2 * (int64_t)kq, xs, row_scale(r < v.R ? rowE[rr] : 0));
  }
}

// ---------------------------------------------------------------- the tensor-core GEMM
struct OzParams {
  int M, N;              // complex extents of C
  int Mpad, NBpad;       // rows of one A' slice / one B'^T slice in the slice buffers
  int kstages;           // K' / OZ_BK
  const int* ea;         // biased exponents per row of A (Mpad)
  const int* eb;         // biased exponents per complex column of B (NBpad / 2)
  cd* C; int64_t c_m, c_n, c_bat;
  cd alpha, beta;
  int* err;              // device error word (bit 1: a wait in this kernel ran out)
  int nprob;             // problems of the batch: problem p's slices start at row p * S * Mpad
                         // (* NBpad) of the tensor maps, its exponents at p * Mpad (* NBpad / 2)
};

template <int S>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    ozgemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzParams P) {
  constexpr int ST = num_stages(S);
  constexpr int SB = stage_bytes(S);
  constexpr int NCOL = tmem_cols(S);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * SB);
  uint64_t* empty = full + ST;
  uint64_t* accum = empty + ST;      // the MMAs of a tile are complete (one commit per tile)
  uint64_t* drained = accum + 1;     // the epilogue has read a tile's accumulators (8 warps arrive)
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(drained + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int tiles_m = P.Mpad / OZ_BM;
  const int tiles_per_prob = tiles_m * (P.NBpad / OZ_BN);
  // this CTA's tiles: blockIdx.x, blockIdx.x + gridDim.x, ... of all problems' tiles
  const int my_tiles = (tiles_per_prob * P.nprob - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  struct Tile {
    int prob, m0, n0;   // n0 in real columns of C'
  };
  auto tile_of = [&](int j) {
    const int t = (int)blockIdx.x + j * (int)gridDim.x;
    const int prob = t / tiles_per_prob, r = t % tiles_per_prob;
    return Tile{prob, (r % tiles_m) * OZ_BM, (r / tiles_m) * OZ_BN};
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(accum, 1);
    mbar_init(drained, OZ_EPI_WARPS);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_holder)),
                 "r"(NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_holder;

  if (warp == 0) {
    // ---- TMA producer: the stage ring runs on across tiles, so the next tile's first stages
    // load while the epilogue drains the current one
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
      asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
      int g = 0;   // stages issued so far (all tiles)
      for (int j = 0; j < my_tiles && !*abort_flag; ++j) {
        const Tile tl = tile_of(j);
        const int yA = tl.prob * S * P.Mpad + tl.m0, yB = tl.prob * S * P.NBpad + tl.n0;
        for (int kb = 0; kb < P.kstages; ++kb, ++g) {
          const int s = g % ST;
          const uint32_t ph = (g / ST) & 1;
          if (!mbar_wait(empty + s, ph ^ 1) || *abort_flag) {
            *abort_flag = 1;
            break;
          }
          unsigned char* st = smem + s * SB;
          mbar_expect_tx(full + s, SB);
#pragma unroll
          for (int i = 0; i < S; ++i) tma_load_2d(st + i * A_TILE, &tmA, full + s, kb * OZ_BK, yA + i * P.Mpad);
#pragma unroll
          for (int i = 0; i < S; ++i)
            tma_load_2d(st + S * A_TILE + i * B_TILE, &tmB, full + s, kb * OZ_BK, yB + i * P.NBpad);
        }
      }
      if (*abort_flag) {
        // let the copies already in flight land before the CTA goes away
        for (int q = (g > ST ? g - ST : 0); q < g; ++q) mbar_wait(full + q % ST, (q / ST) & 1);
      }
    }
  } else if (warp == 1) {
    // ---- MMA issuer: one tile's MMAs after the epilogue has drained the previous tile
    if (lane == 0) {
      int g = 0, commits = 0;
      bool stop = false;
      for (int j = 0; j < my_tiles && !stop; ++j) {
        if (j > 0 && (!mbar_wait(drained, (uint32_t)((j - 1) & 1)) || *abort_flag)) {
          *abort_flag = 1;
          break;
        }
        fence_after();
        for (int kb = 0; kb < P.kstages; ++kb, ++g) {
          const int s = g % ST;
          const uint32_t ph = (g / ST) & 1;
          if (!mbar_wait(full + s, ph) || *abort_flag) {
            *abort_flag = 1;
            stop = true;
            break;
          }
          fence_after();
          const uint32_t st = smem_u32(smem + s * SB);
#pragma unroll
          for (int kk = 0; kk < OZ_BK / 32; ++kk) {
#pragma unroll
            for (int i = 0; i < S; ++i) {
              // Row i of the slice triangle: A_i times B_0 .. B_{S-1-i}.  The B slice tiles of a
              // stage are consecutive 64-row blocks of one swizzled operand, and the level
              // accumulators are consecutive OZ_BN-column blocks of TMEM, so A_i [B_j .. B_{j+n-1}]
              // is one MMA with N = n * OZ_BN whose output columns start at level i + j: the
              // products land in their levels without any per-level MMA.
              const uint64_t ad = smem_desc_sw64(st + i * A_TILE + kk * 32);
              const int nmma = (S - i + OZ_SLICES_PER_MMA - 1) / OZ_SLICES_PER_MMA;
#pragma unroll
              for (int q = 0; q < (S + OZ_SLICES_PER_MMA - 1) / OZ_SLICES_PER_MMA; ++q) {
                if (q >= nmma) break;
                const int jb = q * OZ_SLICES_PER_MMA;
                const int nj = (S - i - jb) < OZ_SLICES_PER_MMA ? (S - i - jb) : OZ_SLICES_PER_MMA;
                const uint64_t bd = smem_desc_sw64(st + S * A_TILE + jb * B_TILE + kk * 32);
                const uint32_t acc = (kb > 0 || kk > 0 || i > 0) ? 1u : 0u;   // i == 0 opens every level
                const uint32_t td = tmem + (uint32_t)((i + jb) * OZ_BN);
                const uint32_t id = idesc_i8(nj * OZ_BN);
                // A_i is shared by the nmma products of this row
                if (nmma == 1) mma_i8<0>(td, ad, bd, id, acc);
                else if (q == 0) mma_i8<1>(td, ad, bd, id, acc);
                else if (q == nmma - 1) mma_i8<3>(td, ad, bd, id, acc);
                else mma_i8<2>(td, ad, bd, id, acc);
              }
            }
          }
          mma_commit(empty + s);   // the stage's smem is free once these MMAs have read it
        }
        mma_commit(accum);         // this tile's MMAs (also those issued before an abort)
        ++commits;
      }
      if (*abort_flag && commits == 0) {
        mma_commit(accum);
        ++commits;
      }
      // no MMA may still write TMEM when it is released
      if (commits > 0) mbar_wait(accum, (uint32_t)((commits - 1) & 1));
    }
  } else if (warp >= 4) {
    // ---- epilogue, eight warps: warp w reads TMEM lanes 32*(w%4) .. +31 (rows m0 + 32*(w%4) +
    // lane, the lane quarter a warp may access) and the 32-column half (w-4)/4 of every level
    const int quarter = warp % 4, half = (warp - 4) / 4;
    const uint32_t tbase = tmem + ((uint32_t)(32 * quarter) << 16);
    const bool use_beta = (P.beta.x != 0.0) || (P.beta.y != 0.0);
    for (int j = 0; j < my_tiles; ++j) {
      const Tile tl = tile_of(j);
      bool ok = true;
      if (lane == 0) ok = mbar_wait(accum, (uint32_t)(j & 1)) && !*abort_flag;   // one poller per warp
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      fence_after();
      if (!ok) {
        *abort_flag = 1;
        break;
      }
      double acc[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) acc[c] = 0.0;
#pragma unroll
      for (int t = S - 1; t >= 0; --t) {
        int v[32];
        __syncwarp();   // tcgen05.ld is warp-collective
        tmem_ld32(tbase + (uint32_t)(t * OZ_BN + half * 32), v);
        const double w = pow2_exact(-7 * (t + 2));
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] += (double)v[c] * w;
      }
      // this warp's reads of the accumulators are complete: the next tile may overwrite them
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(drained);
      const int m = tl.m0 + 32 * quarter + lane;
      if (m < P.M) {
        const int Ea = P.ea[(int64_t)tl.prob * P.Mpad + m];
        const int* eb = P.eb + (int64_t)tl.prob * (P.NBpad / 2);
        cd* Cp = P.C + (int64_t)tl.prob * P.c_bat;
        const int nbase = (tl.n0 + half * 32) / 2;   // first complex column of this half
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int n = nbase + c;
          if (n < P.N) {
            const int Eb = eb[n];
            double re = 0.0, im = 0.0;
            if (Ea > 0 && Eb > 0) {
              const int e = (Ea - 1022) + (Eb - 1022);
              if (e >= -1022 && e <= 1023) {   // one exact power-of-two multiply, as ldexp rounds
                const double sc = pow2_exact(e);
                re = acc[2 * c] * sc;
                im = acc[2 * c + 1] * sc;
              } else {
                re = ldexp(acc[2 * c], e);
                im = ldexp(acc[2 * c + 1], e);
              }
            }
            cd* cp = Cp + (int64_t)m * P.c_m + (int64_t)n * P.c_n;
            cd val = cmul(P.alpha, cmk(re, im));
            if (use_beta) val = cadd(val, cmul(P.beta, *cp));
            *cp = val;
          }
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0 && P.err) atomicOr(P.err, 2);
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(NCOL));
  }
}

// Self-test of the bounded wait: one thread waits on an mbarrier that nothing ever arrives on;
// the wait runs out after limit_ns and the kernel reports it in the error word (bit 2) and
// returns.  Nothing else is in flight, so the context stays usable.
__global__ void wait_probe_kernel(unsigned long long limit_ns, int* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, limit_ns)) atomicOr(err, 4);
}

// ---------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

int get_encoder() {
  std::call_once(g_encode_once, [] {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) {
    set_last_message("cuTensorMapEncodeTiled is not available from the driver");
    return MPSB_ERR_CUDA;
  }
  return MPSB_OK;
}

// 2-d int8 tensor map of a slice buffer (rows of kp bytes), tiles of 64 bytes x box_rows
int make_map(CUtensorMap* map, const int8_t* base, int64_t kp, int64_t rows, int box_rows) {
  cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kp};
  cuuint32_t box[2] = {(cuuint32_t)OZ_BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_message("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return MPSB_ERR_CUDA;
  }
  return MPSB_OK;
}

// SMs of the current device (cached per device)
int device_sm_count() {
  static std::mutex mu;
  static int count[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  std::lock_guard<std::mutex> lock(mu);
  if (count[dev] <= 0 && cudaDeviceGetAttribute(&count[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    count[dev] = 0;
  return count[dev] > 0 ? count[dev] : 148;
}

typedef void (*OzKernel)(CUtensorMap, CUtensorMap, OzParams);
typedef void (*SplitKernel)(SliceView, const int*, int64_t, int8_t*, int64_t, int);
typedef void (*FusedKernel)(SliceView, int*, int64_t, int8_t*, int64_t, int, int);

template <int S>
struct OzTable {
  static OzKernel gemm() { return ozgemm_kernel<S>; }
  static SplitKernel split(bool b) { return b ? oz_split_kernel<S, true> : oz_split_kernel<S, false>; }
  static FusedKernel fused(bool b) { return b ? oz_slice_rows_kernel<S, true> : oz_slice_rows_kernel<S, false>; }
  static int smem() { return smem_bytes(S); }
};

OzKernel pick_gemm(int S) {
  switch (S) {
    case 3: return OzTable<3>::gemm();
    case 4: return OzTable<4>::gemm();
    case 5: return OzTable<5>::gemm();
    case 6: return OzTable<6>::gemm();
    case 7: return OzTable<7>::gemm();
  }
  return nullptr;
}
SplitKernel pick_split(int S, bool b) {
  switch (S) {
    case 3: return OzTable<3>::split(b);
    case 4: return OzTable<4>::split(b);
    case 5: return OzTable<5>::split(b);
    case 6: return OzTable<6>::split(b);
    case 7: return OzTable<7>::split(b);
  }
  return nullptr;
}
FusedKernel pick_fused(int S, bool b) {
  switch (S) {
    case 3: return OzTable<3>::fused(b);
    case 4: return OzTable<4>::fused(b);
    case 5: return OzTable<5>::fused(b);
    case 6: return OzTable<6>::fused(b);
    case 7: return OzTable<7>::fused(b);
  }
  return nullptr;
}
int smem_of(int S) {
  switch (S) {
    case 3: return OzTable<3>::smem();
    case 4: return OzTable<4>::smem();
    case 5: return OzTable<5>::smem();
    case 6: return OzTable<6>::smem();
    case 7: return OzTable<7>::smem();
  }
  return 0;
}

inline int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

}  // namespace

int wait_probe_launch(double seconds, int* err, cudaStream_t s) {
  if (!(seconds > 0.0) || seconds > 10.0 || !err) return MPSB_ERR_INVALID_ARG;
  wait_probe_kernel<<<1, 32, 0, s>>>((unsigned long long)(seconds * 1e9), err);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

bool ozgemm_supported(const Gemm& g, int slices) {
  if (slices < OZ_MIN_SLICES || slices > OZ_MAX_SLICES) return false;
  if (g.batch < 1 || g.batch > 65535 || g.M <= 0 || g.N <= 0 || g.K <= 0) return false;
  // exact int32 accumulation: S * 127^2 * 2K < 2^31
  return (int64_t)slices * 127 * 127 * 2 * (int64_t)g.K < (int64_t(1) << 31);
}

size_t ozgemm_scratch_bytes(const Gemm& g, int slices) {
  const int64_t Mpad = round_up(g.M, OZ_BM), NBpad = round_up(2 * (int64_t)g.N, OZ_BN);
  const int64_t Kp = round_up(2 * (int64_t)g.K, OZ_KP_ALIGN);
  return (size_t)g.batch * ((size_t)slices * (Mpad + NBpad) * Kp + (size_t)(Mpad + NBpad / 2) * sizeof(int)) + 1024;
}

int ozgemm_launch(const Gemm& g, int slices, void* scratch, size_t scratch_bytes, int* err, Workspace* ws,
                  cudaStream_t s) {
  if (!ozgemm_supported(g, slices)) return MPSB_ERR_UNSUPPORTED;
  if (scratch_bytes < ozgemm_scratch_bytes(g, slices)) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(get_encoder());
  const int S = slices;
  const int64_t Mpad = round_up(g.M, OZ_BM), NBpad = round_up(2 * (int64_t)g.N, OZ_BN);
  const int64_t Kp = round_up(2 * (int64_t)g.K, OZ_KP_ALIGN);
  const int64_t B = g.batch;
  if (B * Mpad * S >= (int64_t(1) << 31) || B * NBpad * S >= (int64_t(1) << 31) || Kp >= (int64_t(1) << 31))
    return MPSB_ERR_UNSUPPORTED;
  // scratch: the A slices of every problem [B][S][Mpad][Kp], then the B slices [B][S][NBpad][Kp],
  // then the row exponents [B][Mpad] and the column exponents [B][NBpad / 2]
  int8_t* sa = static_cast<int8_t*>(scratch);
  int8_t* sb = sa + (size_t)B * S * Mpad * Kp;
  int* ea = reinterpret_cast<int*>(sb + (size_t)B * S * NBpad * Kp);
  int* eb = ea + B * Mpad;
  // A' rows = rows m of op(A): element (m, k) at A[m a_m + k a_k]
  SliceView va{g.A, g.M, g.K, g.a_m, g.a_k, g.conjA, g.a_b};
  // B'^T rows come from columns n of op(B): element (n, k) at B[n b_n + k b_k]
  SliceView vb{g.B, g.N, g.K, g.b_n, g.b_k, g.conjB, g.b_b};
  const int kc = (int)(Kp / 2);   // complex k extent covered by the slice grid
  const unsigned bz = (unsigned)B;
  // Rows per CTA of the fused exponent-and-slice kernel: a power of two up to 32 whose rows fit
  // its shared memory, lowered while fewer than about two CTAs per SM would be busy, but not below
  // 8 when the rows are the contiguous index (8 rows of 16 bytes make a full line per column);
  // 0 when that does not fit (the exponent scan and the slicing then run as two kernels).
  // Depends on the problem's shape and layout only.
  auto fused_rows = [&](const SliceView& v, int64_t rows_padded) {
    const int floor_rows = (v.x_r == 1) ? 8 : 1;
    int rpc = 32;
    while (rpc >= floor_rows && (size_t)rpc * (kc + 1) * sizeof(cd) > (size_t)OZ_FUSED_SMEM) rpc /= 2;
    if (rpc < floor_rows) return 0;
    while (rpc > floor_rows && rows_padded * B / rpc < 2 * 148) rpc /= 2;
    return rpc;
  };
  const int ra = fused_rows(va, Mpad), rb = fused_rows(vb, NBpad / 2);
  if (ra == 0 || rb == 0)
    MPSB_CUDA_TRY(cudaMemsetAsync(ea, 0, (size_t)B * (Mpad + NBpad / 2) * sizeof(int), s));
  // k tiles per exponent-scan CTA of the two-kernel form: up to 8 while the grid stays above 8
  // CTAs per SM (the maximum is the same whatever the partition)
  const int ktiles = (g.K + 31) / 32;
  auto kper = [&](int rows) {
    const int64_t tiles = (int64_t)((rows + 31) / 32) * ktiles * B;
    return (int)std::max<int64_t>(1, std::min<int64_t>(8, tiles / (148 * 8)));
  };
  auto slice = [&](const SliceView& v, int* e, int64_t rows_padded, int8_t* dst, int64_t rows_out, bool bmode,
                   int rpc) -> int {
    count_launch(ws);
    if (rpc > 0) {
      FusedKernel fk = pick_fused(S, bmode);
      const int smem = (int)((size_t)rpc * (kc + 1) * sizeof(cd));
      MPSB_TRY(ensure_kernel_attrs((const void*)fk, OZ_FUSED_SMEM));
      fk<<<dim3((unsigned)(rows_padded / rpc), 1, bz), 256, smem, s>>>(v, e, rows_padded, dst, rows_out, (int)Kp, rpc);
      MPSB_CUDA_TRY(cudaGetLastError());
      return MPSB_OK;
    }
    const int kp = kper(v.R);
    oz_rowexp_kernel<<<dim3((unsigned)((v.R + 31) / 32), (unsigned)((ktiles + kp - 1) / kp), bz), 256, 0, s>>>(
        v, e, rows_padded, kp);
    MPSB_CUDA_TRY(cudaGetLastError());
    count_launch(ws);
    pick_split(S, bmode)<<<dim3((unsigned)(rows_padded / 32), (unsigned)(kc / 32), bz), 256, 0, s>>>(
        v, e, rows_padded, dst, rows_out, (int)Kp);
    MPSB_CUDA_TRY(cudaGetLastError());
    return MPSB_OK;
  };
  MPSB_TRY(slice(va, ea, Mpad, sa, Mpad, false, ra));
  MPSB_TRY(slice(vb, eb, NBpad / 2, sb, NBpad, true, rb));

  CUtensorMap ta, tb;
  MPSB_TRY(make_map(&ta, sa, Kp, B * S * Mpad, OZ_BM));
  MPSB_TRY(make_map(&tb, sb, Kp, B * S * NBpad, OZ_BN));
  OzParams P;
  P.M = g.M; P.N = g.N; P.Mpad = (int)Mpad; P.NBpad = (int)NBpad; P.kstages = (int)(Kp / OZ_BK);
  P.ea = ea; P.eb = eb;
  P.C = g.C; P.c_m = g.c_m; P.c_n = g.c_n; P.c_bat = g.c_b; P.alpha = g.alpha; P.beta = g.beta;
  P.err = err;
  OzKernel fn = pick_gemm(S);
  MPSB_TRY(ensure_kernel_attrs((const void*)fn, smem_of(S)));
  const int64_t tiles = (Mpad / OZ_BM) * (NBpad / OZ_BN) * B;   // output tiles of all problems
  if (tiles >= (int64_t(1) << 31)) return MPSB_ERR_UNSUPPORTED;
  P.nprob = (int)B;
  const int grid = (int)std::min<int64_t>(tiles, device_sm_count());   // one persistent CTA per SM
  count_launch(ws);
  Workspace::TimedLaunch ev{nullptr, nullptr, 0.0};
  const bool timed = ws && ws->prof && !ws->capturing;
  if (timed) {
    MPSB_CUDA_TRY(cudaEventCreate(&ev.start));
    MPSB_CUDA_TRY(cudaEventCreate(&ev.stop));
    MPSB_CUDA_TRY(cudaEventRecord(ev.start, s));
    // S(S+1)/2 slice products of the real (M x 2K) x (2K x 2N) GEMM per problem, 2 ops per MAC
    ev.ops = 2.0 * (S * (S + 1) / 2) * (double)g.M * (2.0 * g.N) * (2.0 * g.K) * (double)B;
  }
  fn<<<dim3((unsigned)grid), OZ_THREADS, smem_of(S), s>>>(ta, tb, P);
  MPSB_CUDA_TRY(cudaGetLastError());
  if (timed) {
    MPSB_CUDA_TRY(cudaEventRecord(ev.stop, s));
    ws->prof->push_back(ev);
  }
  return MPSB_OK;
}

}  // namespace mpsb
