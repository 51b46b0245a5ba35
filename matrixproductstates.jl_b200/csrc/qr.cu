// Householder QR with the LAPACK zgeqrf + zungqr conventions (the routines qrq! calls,
// src/orthonormalisation.jl:180-184), Q (and optionally R) of an m x n complex matrix, m >= n.
//
// Reflector convention (zlarfg): for column j with alpha = A[j,j] and x = A[j+1:m, j],
//   if x == 0 and Im(alpha) == 0:  tau = 0 (H = I, R[j,j] = alpha)
//   else beta = -copysign(|(alpha, x)|, Re alpha), tau = (beta - alpha)/beta,
//        v = [1; x/(alpha - beta)], R[j,j] = beta (real)
// H(j)^H = I - conj(tau) v v^H is applied to the trailing columns (zgeqr2), and
// Q = H(1)...H(n) [I; 0] (zungqr).  Only the span of Q carries physics in the sweeps; the
// sign / phase rule above is what must match LAPACK, and it also fixes the "junk" columns of
// zero-padded (rank-deficient) sites.
//
// Range: the sums behind |x|, v^H a and V^H x are taken on x scaled by 2^-e, e the binary
// exponent of the largest |Re|, |Im| of x when that lies outside [2^-256, 2^257) and 0 inside
// (each CTA its own e; the partials are brought to the largest e on combination), and the
// reflector is formed on (alpha, x) scaled by 2^-E, E the larger of that exponent and alpha's
// (taken the same way).  Inside the range nothing is scaled: the instruction stream is the
// plain formula's.  Outside it the scalings are exact powers of two, so columns whose norm is
// near or below sqrt(DBL_MIN) (amplitudes of 1e-150 and smaller occur in the sweeps from
// product states) get the reflector zlarfg's safe-minimum rescaling gives them instead of an
// overflow.  Not covered: an unscaled column's products with entries below 2^-766 of another
// column underflow (LAPACK's normalised v keeps them), i.e. spreads of more than ~1e-230
// between the columns of one matrix lose those small columns' directions.
//
// B200 mapping: one thread-block cluster per matrix, rows split over its C CTAs (32*RPL
// rows each; the whole matrix lives in distributed shared memory).  Blocked right-looking
// algorithm with panels of NB columns.  Every exchange between CTAs is a *push*: the
// producer writes its values straight into each consumer's shared memory with st.async,
// whose completion is counted in bytes on the consumer's mbarrier; the consumer waits on
// its own mbarrier (bounded) and then reads only local shared memory.  No cluster-wide
// barrier sits inside the loops.
//   * column j: each warp reduces its panel columns over the CTA's rows with warp shuffles
//     (lane = row) and pushes the sums to all C CTAs; the owner of row j pushes that row;
//     after the wait warp 0 forms the reflector, w = v^H A and the new column of the
//     compact-WY factor T, and every warp updates its columns;
//   * trailing columns: partials of V^H A pushed to the owner of each column slice,
//     reduced there in a fixed order with T^H applied, the slice pushed to every CTA,
//     then A -= V W locally.
// The cluster kernel ends with R, the explicit reflectors V (m x n, unit lower trapezoidal)
// and tau in global memory, and E = [I; 0] in Q.  Q is then formed on the whole GPU with the
// UT-transform identity  Q = (I - V T V^H) E = E - V (T V1^H),  T^{-1} = diag(1/tau) +
// striu(V^H V)  (V1 = top n x n block of V): a tensor-core GEMM for G = V^H V, one
// back-substitution kernel for M = T V1^H (T^{-1} M = V1^H, so M[i,:] = tau_i (V1^H[i,:] -
// sum_{k>i} G[i,k] M[k,:]) needs no division and gives M[i,:] = 0 when tau_i = 0), and a
// tensor-core GEMM for Q -= V M.  In exact arithmetic this is zungqr's Q.
// Reductions run in a fixed order, so every CTA computes bit-identical reflectors and
// results are reproducible run to run.  Each wait gives up after a bounded number of polls,
// records the timeout in the error word and lets the kernel run to completion.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "workspace.cuh"

namespace cg = cooperative_groups;

namespace mpsb {
namespace {

constexpr int NT = 256, NW = 8;
constexpr int CMAX = 16;
constexpr size_t SMEM_LIMIT = 227 * 1024;
constexpr int WAIT_LIMIT = 1 << 22;
enum { MB_COL0 = 0, MB_COL1, MB_RS, MB_AG, MB_COUNT };

struct QrParams {
  QrProblem p;
  cd* V;     // [batch][n][m] explicit unit lower trapezoidal reflectors (output)
  cd* Tg;    // [batch][npanels][NB][NB] compact-WY factor of every panel (output)
  int C, npanels, ldS, ksmax;
  // shared-memory offsets (complex elements) and the byte offset of the mbarriers
  int o_S, o_rcol, o_rrs, o_w2s, o_rag, o_T, o_bc, o_tst, o_mbar;
};

// ---- PTX helpers -------------------------------------------------------------------
__device__ __forceinline__ uint32_t su32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
// 16-byte remote store into CTA-rank-mapped shared memory, completion counted on its mbarrier
__device__ __forceinline__ void st_async(uint32_t raddr, cd v, uint32_t rmbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];"
               ::"r"(raddr), "d"(v.x), "d"(v.y), "r"(rmbar) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait of the whole CTA on the phase of the given parity.  Only thread 0 polls --
// polling warps would compete with the computing warps for the shared-memory pipe -- and the
// block barrier then publishes the completion (and the pushed data) to every thread.  A
// timeout is recorded in the error word and later waits are skipped.
__device__ __forceinline__ void cta_wait(uint32_t mbar, uint32_t parity, bool& failed, int* err) {
  if (threadIdx.x == 0 && !failed) {
    int it = 0;
    while (!mbar_test(mbar, parity)) {
      if (++it >= WAIT_LIMIT) {
        failed = true;
        if (err) atomicOr(err, 1);
        break;
      }
    }
  }
  __syncthreads();
}

// sum of the C partials part[q*stride] in a fixed order (tree over the ranks, independent loads)
__device__ __forceinline__ cd sum_ranks(const cd* part, int stride, int C) {
  cd v[CMAX];
#pragma unroll
  for (int q = 0; q < CMAX; ++q) v[q] = (q < C) ? part[q * stride] : cmk(0.0, 0.0);
#pragma unroll
  for (int w = CMAX / 2; w > 0; w >>= 1)
#pragma unroll
    for (int q = 0; q < w; ++q) v[q] = cadd(v[q], v[q + w]);
  return v[0];
}

// The exponent slot of a rank's column message: no nonzero entry below the diagonal.
constexpr int ESENT = -100000;

// 2^k for -1022 <= k <= 1023, written into the exponent field
__device__ __forceinline__ double pow2i(int k) { return __hiloint2double((k + 1023) << 20, 0); }
// 2^k for k <= 0; 0 below the normal range (a contribution 2^-1022 times smaller than the rest)
__device__ __forceinline__ double pow2neg(int k) { return k >= -1022 ? pow2i(k) : 0.0; }
// binary exponent (clamped to [-1022, 1022]) of a nonnegative double from its high word;
// high word 0 (|v| < 2^-1042) is the caller's "zero"
__device__ __forceinline__ int expo_hi(unsigned hi) {
  const int b = (int)((hi >> 20) & 0x7ffu);
  return min(max(b, 1) - 1023, 1022);
}
__device__ __forceinline__ cd cscal(cd v, double f) { return cmk(v.x * f, v.y * f); }

// Half-width of the binary-exponent window [2^-SWIN, 2^(SWIN+1)) inside which nothing is scaled.
constexpr int SWIN = 256;
constexpr double WHI = 0x1p256, WLO = 0x1p-256;   // 2^SWIN, 2^-SWIN
static_assert(SWIN == 256, "WHI / WLO follow SWIN");

// A CTA whose partials are those of x 2^-e sends its |x|^2 partial (real) in the imaginary
// part and a quiet NaN carrying SCODE + e in the real part, so the unscaled combination of the
// ranks is NaN exactly when some rank scaled.
constexpr long long SCODE = 4096;
__device__ __forceinline__ double scale_nan(int e) {
  return __longlong_as_double(0x7ff8000000000000ll | (unsigned long long)(SCODE + e));
}
__device__ __forceinline__ int scale_of_nan(double v) { return (int)((__double_as_longlong(v) & 0xffffll) - SCODE); }

// The reflector when some rank scaled its partials or alpha lies outside the unit range (rare:
// kept out of line so the common path's instructions stay the plain formula's).  Lane c < pw
// of warp 0 gets s = its combined partial at the scale 2^-E (lane jl: |x|^2 at 2^-2E), and
// every lane tau, beta, rs = 1/(alpha - beta) at 2^-E, and fE = 2^-E.  Returned by value, so
// the caller's variables stay in registers on the common path.
struct Reflector {
  cd s, tau, beta, rs;
  double fE;
};
__device__ __noinline__ Reflector reflector_scaled(const cd* rb, int RS, int C, int lane, int jl, int pw, cd alpha) {
  Reflector o;
  int e[CMAX];
  int ex = ESENT;
#pragma unroll
  for (int q = 0; q < CMAX; ++q) {
    e[q] = ESENT;
    if (q < C) {
      const cd pq = rb[q * RS + jl];
      e[q] = pq.x != pq.x ? scale_of_nan(pq.x) : (pq.x != 0.0 ? 0 : ESENT);
    }
    ex = max(ex, e[q]);
  }
  cd v = cmk(0.0, 0.0);
  if (lane < pw) {
    const int mult = lane == jl ? 2 : 1;
#pragma unroll
    for (int q = 0; q < CMAX; ++q) {
      if (q >= C || e[q] == ESENT) continue;
      cd pq = rb[q * RS + lane];
      if (lane == jl) pq = cmk(pq.x != pq.x ? pq.y : pq.x, 0.0);
      v = cadd(v, cscal(pq, pow2neg(mult * (e[q] - ex))));
    }
  }
  const double xn2x = __shfl_sync(0xffffffffu, v.x, jl);   // |x|^2 2^-2ex
  const unsigned ha = (unsigned)__double2hiint(fmax(fabs(alpha.x), fabs(alpha.y)));
  int ea = expo_hi(ha);
  ea = (ha == 0u) ? ESENT : (ea >= -SWIN && ea <= SWIN ? 0 : ea);
  const int E = max(ex, ea);   // not both ESENT: x == 0 with real alpha never gets here
  o.fE = pow2i(-E);
  const cd as = cscal(alpha, o.fE);
  const double xn2 = (ex == ESENT) ? 0.0 : xn2x * pow2neg(2 * (ex - E));
  const double nrm = sqrt(as.x * as.x + as.y * as.y + xn2);
  const double b = -copysign(nrm, alpha.x);
  const double dr = as.x - b;
  const double ib = 1.0 / b;
  const double id = 1.0 / (dr * dr + as.y * as.y);
  o.tau = cmk((b - as.x) * ib, -as.y * ib);
  o.beta = cmk(b * pow2i(E), 0.0);
  o.rs = cmk(dr * id, -as.y * id);
  o.s = (ex == ESENT) ? cmk(0.0, 0.0) : cscal(v, pow2neg(ex - E));
  return o;
}

__device__ __forceinline__ cd shfl(cd v, int src) {
  return cmk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
// ---- per-CTA shared memory map (complex elements) -------------------------------------
// S     [(ROWS+1) * n]       this CTA's rows, column-major, ld = ROWS+1
// rcol  [2][C][2*NB]         column exchange (two parities): pq from each rank, row j from its owner
// rrs   [C][NB*ksmax]        partials of V^H A received from each rank for my column slice
// w2s   [NB*ksmax]           my reduced slice
// rag   [NB*n]               the gathered W2 (all slices)
// T     [NB*NB]              compact-WY factor of the current panel (column-major NB x NB)
// mbar  [MB_COUNT] u64

// V[r, i] of panel p0 for global row g (unit lower trapezoidal, stored below the diagonal)
#define VAL_V(g, i, rr) ((g) == p0 + (i) ? cmk(1.0, 0.0) : S[(p0 + (i)) * ldS + (rr)])

// Partial sums W[i, k] = sum over this CTA's rows of conj(V[r, i]) A[r, kb + k] for the panel at
// p0 (width pw), pushed with st.async to the owner of column slice k / KS.  Threads t in
// [0, nthr) take (k, half panel) pairs; the rows of the panel's diagonal block (where V is 1 or
// 0 above its stored part) are handled apart so the bulk loop carries no per-element tests.
template <int ROWS, int NB>
__device__ __forceinline__ void partials_push(const cd* S, int ldS, cd* rrs, uint32_t mb_rs, int crank, int ksmax,
                                              int row0, int m, int p0, int pw, int kb, int nt, int KS, int t,
                                              int nthr) {
  const int lo = max(0, p0 - row0), hi = min(ROWS, m - row0);
  const int mid = min(hi, max(lo, p0 + pw - row0));
  for (int e = t; e < 2 * nt; e += nthr) {
    const int k = e % nt, i0 = (e / nt) * (NB / 2);
    const int iv = min(NB / 2, pw - i0);   // valid panel columns in this half
    cd acc[NB / 2];
#pragma unroll
    for (int i = 0; i < NB / 2; ++i) acc[i] = cmk(0.0, 0.0);
    const cd* Ak = S + (kb + k) * ldS;
    for (int rr = lo; rr < mid; ++rr) {
      const int g = row0 + rr;
      const cd a = Ak[rr];
#pragma unroll
      for (int i = 0; i < NB / 2; ++i) {
        const int ii = i0 + i;
        if (i < iv && g >= p0 + ii) cfma_cj(acc[i], VAL_V(g, ii, rr), a);
      }
    }
    for (int rr = mid; rr < hi; ++rr) {
      const cd a = Ak[rr];
#pragma unroll
      for (int i = 0; i < NB / 2; ++i)
        if (i < iv) cfma_cj(acc[i], S[(p0 + i0 + i) * ldS + rr], a);
    }
    const int so = k / KS, kk = k - so * KS;
    const uint32_t rm = mapa(mb_rs, so);
#pragma unroll
    for (int i = 0; i < NB / 2; ++i)
      if (i < iv) st_async(mapa(su32(&rrs[crank * NB * ksmax + (i0 + i) + NB * kk]), so), acc[i], rm);
  }
}

// Row `rr` of the panel's V (zero above its diagonal block and outside the matrix), in registers.
template <int NB>
__device__ __forceinline__ void load_vrow(cd (&v)[NB], const cd* S, int ldS, int rr, int g, int m, int p0, int pw) {
#pragma unroll
  for (int i = 0; i < NB; ++i)
    v[i] = (i < pw && g >= p0 + i && g < m) ? VAL_V(g, i, rr) : cmk(0.0, 0.0);
}

template <int RPL, int NB>
__global__ void __launch_bounds__(NT, 1) qr_kernel(QrParams P) {
  constexpr int ROWS = 32 * RPL;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* sm = reinterpret_cast<cd*>(smem_raw);
  const int C = P.C, ldS = P.ldS, ksmax = P.ksmax;
  const int m = P.p.m, n = P.p.n;
  const int crank = (int)cluster.block_rank();
  const int prob = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int row0 = crank * ROWS;
  int* err = P.p.err;

  cd* S = sm + P.o_S;
  cd* rcol = sm + P.o_rcol;
  cd* rrs = sm + P.o_rrs;
  cd* w2s = sm + P.o_w2s;
  cd* rag = sm + P.o_rag;
  cd* Tall = sm + P.o_T;
  cd* bcs = sm + P.o_bc;        // tau, beta, 1/(alpha - beta) at scale 2^-E, and 2^-E of the current column
  cd* bcw = bcs + 4;            // w_c of the current column
  cd* tst = sm + P.o_tst;       // tst[jl*NB + c] = t_c (c < jl), tst[jl*NB + jl] = tau_jl
  uint64_t* mb = reinterpret_cast<uint64_t*>(smem_raw + P.o_mbar);
  uint32_t mbs[MB_COUNT];
#pragma unroll
  for (int k = 0; k < MB_COUNT; ++k) mbs[k] = su32(&mb[k]);
  uint32_t ph[MB_COUNT];
#pragma unroll
  for (int k = 0; k < MB_COUNT; ++k) ph[k] = 0;
  bool failed = false;

  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < MB_COUNT; ++k) mbar_init(mbs[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {  // ---- load this CTA's rows
    const cd* X = P.p.X + (int64_t)prob * P.p.x_b;
    for (int e = tid; e < ROWS * n; e += NT) {
      int rr = e % ROWS, cc = e / ROWS, g = row0 + rr;
      S[cc * ldS + rr] = (g < m) ? X[(int64_t)g * P.p.x_r + (int64_t)cc * P.p.x_c] : cmk(0.0, 0.0);
    }
  }
  cluster.sync();   // mbarriers initialised cluster-wide before any push

  // ================================ factorisation ================================
  int sp = 0;
  for (int pi = 0; pi < P.npanels; ++pi) {
    const int p0 = pi * NB;
    const int pw = min(NB, n - p0);
    for (int jl = 0; jl < pw; ++jl) {
      const int j = p0 + jl;
      constexpr int RS = 2 * NB;   // per rank: NB sums, NB owner-row values
      cd* rb = rcol + sp * (C * RS);
      const uint32_t mbc = mbs[MB_COL0 + sp];
      const int owner = j / ROWS;
      // -- phase A: partial sums over this CTA's rows g > j, pushed to every CTA
      cd x[RPL];
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        int r = lane + 32 * q, g = row0 + r;
        x[q] = (g > j && g < m) ? S[j * ldS + r] : cmk(0.0, 0.0);
      }
      {  // this warp's (at most two) panel columns c0 = warp, c1 = warp + NW, reduced together
        static_assert(NB <= 2 * NW, "at most two panel columns per warp");
        const int c0 = warp, c1 = warp + NW;
        cd a0 = cmk(0.0, 0.0), a1 = cmk(0.0, 0.0);
        double mx = 0.0;   // largest |Re|, |Im| of x over this CTA's rows (every warp finds the same)
#pragma unroll
        for (int q = 0; q < RPL; ++q) mx = fmax(mx, fmax(fabs(x[q].x), fabs(x[q].y)));
        const unsigned hb = __reduce_max_sync(0xffffffffu, (unsigned)__double2hiint(mx));
        auto partials = [&](const cd (&xv)[RPL]) {
#pragma unroll
          for (int q = 0; q < RPL; ++q) {
            const int r = lane + 32 * q;
            if (c0 < pw) {
              const cd a = S[(p0 + c0) * ldS + r];
              if (c0 == jl)     cfma_cj(a0, xv[q], xv[q]);   // |x|^2
              else if (c0 > jl) cfma_cj(a0, xv[q], a);       // conj(x) a
              else              cfma_cj(a0, a, xv[q]);       // conj(a) x  (V^H x for the T column)
            }
            if (c1 < pw) {
              const cd a = S[(p0 + c1) * ldS + r];
              if (c1 == jl)     cfma_cj(a1, xv[q], xv[q]);
              else if (c1 > jl) cfma_cj(a1, xv[q], a);
              else              cfma_cj(a1, a, xv[q]);
            }
          }
        };
        auto reduce = [&]() {
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            a0.x += __shfl_xor_sync(0xffffffffu, a0.x, off);
            a0.y += __shfl_xor_sync(0xffffffffu, a0.y, off);
            a1.x += __shfl_xor_sync(0xffffffffu, a1.x, off);
            a1.y += __shfl_xor_sync(0xffffffffu, a1.y, off);
          }
        };
        partials(x);
        reduce();
        // this CTA's scale 2^-e: e = 0 inside the window (the sums above stand), else mx's
        // binary exponent, and the sums are redone on x 2^-e (ESENT: x == 0, or below 2^-1042)
        const int ee = expo_hi(hb);
        const int e_loc = (hb == 0u) ? ESENT : (ee >= -SWIN && ee <= SWIN ? 0 : ee);
        if (e_loc != 0 && e_loc != ESENT) {
          const double f = pow2i(-e_loc);
          cd xs[RPL];
#pragma unroll
          for (int q = 0; q < RPL; ++q) xs[q] = cscal(x[q], f);
          a0 = a1 = cmk(0.0, 0.0);
          partials(xs);
          reduce();
        }
        if (lane < C) {
          const uint32_t rm = mapa(mbc, lane);
          if (e_loc != 0 && e_loc != ESENT) {
            if (c0 == jl) a0 = cmk(scale_nan(e_loc), a0.x);
            if (c1 == jl) a1 = cmk(scale_nan(e_loc), a1.x);
          }
          if (c0 < pw) st_async(mapa(su32(&rb[crank * RS + c0]), lane), a0, rm);
          if (c1 < pw) st_async(mapa(su32(&rb[crank * RS + c1]), lane), a1, rm);
        }
      }
      if (crank == owner && warp == NW - 1 && lane < pw) {
        const cd v = S[(p0 + lane) * ldS + (j - row0)];
        for (int q = 0; q < C; ++q) st_async(mapa(su32(&rb[crank * RS + NB + lane]), q), v, mapa(mbc, q));
      }
      if (tid == 0) mbar_expect(mbc, (uint32_t)((C + 1) * pw * sizeof(cd)));
      cta_wait(mbc, ph[MB_COL0 + sp], failed, err);
      ph[MB_COL0 + sp] ^= 1;
      // -- phase B: warp 0 forms the reflector from the gathered sums (local reads only) and
      // publishes tau / beta / scale, w_c (c > jl) and t_c (c < jl, for T at panel end)
      if (warp == 0) {
        cd s = cmk(0.0, 0.0), rj = cmk(0.0, 0.0);
        if (lane < pw) {
          s = sum_ranks(rb + lane, RS, C);
          rj = rb[owner * RS + NB + lane];
        }
        const cd alpha = shfl(rj, jl);
        const double xn2 = __shfl_sync(0xffffffffu, s.x, jl);   // NaN: some rank scaled its partials
        const double am = fabs(alpha.x) + fabs(alpha.y);   // alpha's window: (2^-SWIN, 2^SWIN)
        cd tau, beta, rs;
        double fE = 1.0;
        if (xn2 == 0.0 && alpha.y == 0.0) {   // x == 0 (an unscaled nonzero x has |x|^2 >= 2^-2SWIN)
          tau = cmk(0.0, 0.0); beta = alpha; rs = cmk(1.0, 0.0);
        } else if (xn2 >= 0.0 && am < WHI && (xn2 > 0.0 || am > WLO)) {
          // tau = (beta - alpha)/beta and rs = 1/(alpha - beta) from two independent
          // reciprocals, 1/beta and 1/|alpha - beta|^2 (Re(alpha) - beta has no cancellation:
          // beta carries the opposite sign of Re(alpha))
          const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
          const double b = -copysign(nrm, alpha.x);
          const double dr = alpha.x - b;
          const double ib = 1.0 / b;
          const double id = 1.0 / (dr * dr + alpha.y * alpha.y);
          tau = cmk((b - alpha.x) * ib, -alpha.y * ib);
          beta = cmk(b, 0.0);
          rs = cmk(dr * id, -alpha.y * id);
        } else {
          const Reflector o = reflector_scaled(rb, RS, C, lane, jl, pw, alpha);
          s = o.s; tau = o.tau; beta = o.beta; rs = o.rs; fE = o.fE;
        }
        // w_c = a_c[j] + conj(rs) (x 2^-E)^H a_c and t_c = conj(V[j, c]) + rs V[:, c]^H (x 2^-E)
        if (lane > jl && lane < pw) bcw[lane] = cadd(rj, cmul(cconj(rs), s));
        else if (lane < jl) tst[jl * NB + lane] = cadd(cconj(rj), cmul(rs, s));
        if (lane == 0) { bcs[0] = tau; bcs[1] = beta; bcs[2] = rs; bcs[3] = cmk(fE, 0.0); tst[jl * NB + jl] = tau; }
      }
      __syncthreads();
      const cd tau = bcs[0], beta = bcs[1], rs = bcs[2];
      const double fE = bcs[3].x;
      if ((tau.x != 0.0) || (tau.y != 0.0)) {
        cd vr[RPL];
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
          int g = row0 + lane + 32 * q;
          vr[q] = (g == j) ? cmk(1.0, 0.0) : cmul(rs, fE == 1.0 ? x[q] : cscal(x[q], fE));   // x is 0 above j and in padding
        }
        const cd ctau = cconj(tau);
        if (warp == (jl % NW)) {
#pragma unroll
          for (int q = 0; q < RPL; ++q) {
            int r = lane + 32 * q, g = row0 + r;
            if (g == j) S[j * ldS + r] = beta;
            else if (g > j && g < m) S[j * ldS + r] = vr[q];
          }
        }
        for (int c = warp; c < pw; c += NW) {
          if (c > jl) {
            const cd f = cmul(ctau, bcw[c]);
#pragma unroll
            for (int q = 0; q < RPL; ++q) {
              int r = lane + 32 * q, g = row0 + r;
              if (g >= j && g < m) {
                cd* a = &S[(p0 + c) * ldS + r];
                *a = csub(*a, cmul(f, vr[q]));
              }
            }
          }
        }
      }
      __syncthreads();
      sp ^= 1;
    }
    cd* Tp = Tall;   // the previous panel's T was last read before its all-gather wait
    // T (compact WY, zlarft forward/columnwise) from the stashed t vectors, by warp 0 while the
    // other warps start on the trailing partials: T[0:jl, jl] = -tau_jl T[0:jl, 0:jl] t_jl
    if (warp == 0) {
      for (int jl = 0; jl < pw; ++jl) {
        const cd tj = tst[jl * NB + jl];
        cd a4[4] = {cmk(0.0, 0.0), cmk(0.0, 0.0), cmk(0.0, 0.0), cmk(0.0, 0.0)};
#pragma unroll
        for (int c = 0; c < NB; ++c)   // T[lane, c] = 0 for c < lane, so c starts at 0 harmlessly
          if (c < jl && lane < jl) cfma(a4[c & 3], Tp[lane + NB * c], tst[jl * NB + c]);
        const cd acc = cadd(cadd(a4[0], a4[1]), cadd(a4[2], a4[3]));
        if (lane < NB) Tp[lane + NB * jl] = (lane < jl) ? cmul(cmk(-tj.x, -tj.y), acc) : (lane == jl ? tj : cmk(0.0, 0.0));
        __syncwarp();
      }
      if (crank == 0 && lane < NB) {   // lane-owned entries of T, zero outside the panel width
        cd* Tout = P.Tg + ((int64_t)prob * P.npanels + pi) * NB * NB;
        for (int jl = 0; jl < NB; ++jl)
          Tout[lane + NB * jl] = (lane < pw && jl < pw) ? Tp[lane + NB * jl] : cmk(0.0, 0.0);
      }
    }

    // -- trailing update A_t := (I - V T^H V^H) A_t
    const int nt = n - p0 - pw;
    if (nt > 0) {
      const int kb = p0 + pw;
      const int KS = (nt + C - 1) / C;
      const int k0 = crank * KS, ks_mine = max(0, min(nt, k0 + KS) - k0);
      // partials W[i, k] = sum_{my rows} conj(V[r, i]) A[r, k], pushed to the slice owner of k
      if (warp > 0) partials_push<ROWS, NB>(S, ldS, rrs, mbs[MB_RS], crank, ksmax, row0, m, p0, pw, kb, nt, KS,
                                            tid - 32, NT - 32);
      __syncthreads();   // T complete before W2 = T^H W
      if (tid == 0) mbar_expect(mbs[MB_RS], (uint32_t)(C * pw * ks_mine * sizeof(cd)));
      cta_wait(mbs[MB_RS], ph[MB_RS], failed, err);
      ph[MB_RS] ^= 1;
      for (int e = tid; e < pw * ks_mine; e += NT) {
        const int i = e % pw, kk = e / pw;
        cd s = cmk(0.0, 0.0);
        s = sum_ranks(rrs + i + NB * kk, NB * ksmax, C);
        w2s[i + NB * kk] = s;
      }
      __syncthreads();
      // W2 = T^H W on my slice, pushed to every CTA
      for (int e = tid; e < pw * ks_mine; e += NT) {
        const int i = e % pw, kk = e / pw;
        cd s = cmk(0.0, 0.0);
        for (int i2 = 0; i2 <= i; ++i2) cfma_cj(s, Tp[i2 + NB * i], w2s[i2 + NB * kk]);
        const uint32_t la = su32(&rag[i + NB * (k0 + kk)]);
        for (int q = 0; q < C; ++q) st_async(mapa(la, q), s, mapa(mbs[MB_AG], q));
      }
      if (tid == 0) mbar_expect(mbs[MB_AG], (uint32_t)(pw * nt * sizeof(cd)));
      cta_wait(mbs[MB_AG], ph[MB_AG], failed, err);
      ph[MB_AG] ^= 1;
      // A[r, k] -= sum_i V[r, i] W2[i, k]: thread = (row, column group), its V row in registers
      {
        constexpr int G = NT / ROWS;
        const int rr = tid % ROWS, grp = tid / ROWS, g = row0 + rr;
        if (g >= p0 && g < m) {
          cd v[NB];
          load_vrow<NB>(v, S, ldS, rr, g, m, p0, pw);
          for (int k = grp; k < nt; k += G) {
            cd acc = cmk(0.0, 0.0);
#pragma unroll
            for (int i = 0; i < NB; ++i)
              if (i < pw) cfma(acc, v[i], rag[i + NB * k]);
            cd* a = &S[(kb + k) * ldS + rr];
            *a = csub(*a, acc);
          }
        }
      }
      __syncthreads();
    }
  }

  // ---- optional R (rows < n)
  if (P.p.R) {
    cd* Rout = P.p.R + (int64_t)prob * P.p.r_b;
    for (int e = tid; e < ROWS * n; e += NT) {
      int rr = e % ROWS, k = e / ROWS, g = row0 + rr;
      if (g >= n) continue;
      Rout[(int64_t)g * P.p.r_r + (int64_t)k * P.p.r_c] = (k >= g) ? S[k * ldS + rr] : cmk(0.0, 0.0);
    }
  }
  {  // ---- V (unit lower trapezoidal, explicit), tau, and E = [I; 0] into Q (this CTA's rows)
    cd* V = P.V + (int64_t)prob * m * n;
    cd* Q = P.p.Q + (int64_t)prob * P.p.q_b;
    for (int e = tid; e < ROWS * n; e += NT) {
      int rr = e % ROWS, cc = e / ROWS, g = row0 + rr;
      if (g >= m) continue;
      V[g + (int64_t)cc * m] = g < cc ? cmk(0.0, 0.0) : (g == cc ? cmk(1.0, 0.0) : S[cc * ldS + rr]);
      Q[(int64_t)g * P.p.q_r + (int64_t)cc * P.p.q_c] = cmk(g == cc ? 1.0 : 0.0, 0.0);
    }
  }
  // no CTA leaves while a peer may still address its shared memory
  cluster.sync();
}
#undef VAL_V

typedef void (*QrKernel)(QrParams);

template <int NB>
QrKernel kernel_rpl(int rpl) {
  switch (rpl) {
    case 1: return qr_kernel<1, NB>;
    case 2: return qr_kernel<2, NB>;
    case 4: return qr_kernel<4, NB>;
    default: return nullptr;
  }
}

QrKernel kernel_for(int rpl, int nb) {
  if (nb == 16) return kernel_rpl<16>(rpl);
  if (nb == 8) return kernel_rpl<8>(rpl);
  if (nb == 4) return kernel_rpl<4>(rpl);
  return nullptr;
}

size_t layout(QrParams& P, int n, int C, int rows, int nb) {
  P.C = C;
  P.npanels = (n + nb - 1) / nb;
  P.ldS = rows + 1;
  P.ksmax = (n + C - 1) / C;
  int o = 0;
  P.o_S = o;     o += P.ldS * n;
  P.o_rcol = o;  o += 2 * C * 2 * nb;
  P.o_rrs = o;   o += C * nb * P.ksmax;
  P.o_w2s = o;   o += nb * P.ksmax;
  P.o_rag = o;   o += nb * n;
  P.o_T = o;     o += nb * nb;
  P.o_bc = o;    o += 4 + nb;        // tau, beta, rs, 2^-E; w[nb]
  P.o_tst = o;   o += nb * nb;       // t vectors (and tau) of the panel's columns
  P.o_mbar = o * (int)sizeof(cd);
  return (size_t)P.o_mbar + MB_COUNT * sizeof(uint64_t);
}

// ---- M = T V1^H by block back substitution over the panels.  T^{-1} = diag(1/tau) +
// striu(V^H V) is block upper triangular and its diagonal blocks are the inverses of the
// panels' compact-WY factors T_p, so with G = V^H V and B = V1^H (upper triangular):
//   M_p = T_p (B_p - sum_{q > p} G_pq M_q),  p = last panel .. 0.
// One warp per column c of M (M is upper triangular: rows <= c), lanes over rows
// (r = lane + 32 q), holding y = B[:, c] minus the updates so far.  Per panel: the panel's
// rows of y are broadcast by shuffles, M_p = T_p y_p lands in the lanes of those rows, and
// y -= G[:, panel] M_p updates the rows above.  The needed columns of G are staged in shared
// memory one panel ahead (cp.async, double-buffered); the panels' T_p are staged once.
constexpr int TR_WARPS = 8;

template <int QMAX, bool STAGE>
__global__ void __launch_bounds__(32 * TR_WARPS) qr_tmat_kernel(int m, int n, int nb, const cd* __restrict__ Vg,
                                                                 const cd* __restrict__ Tg,
                                                                 const cd* __restrict__ Gg, cd* __restrict__ Mg) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* Gs = reinterpret_cast<cd*>(smem_raw);   // [2][nb][n]
  cd* Ts = Gs + 2 * nb * n;                    // [npan][nb][nb]
  const int prob = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int npan = (n + nb - 1) / nb;
  const cd* V = Vg + (int64_t)prob * m * n;
  const cd* T = Tg + (int64_t)prob * npan * nb * nb;
  const cd* G = Gg + (int64_t)prob * n * n;
  cd* M = Mg + (int64_t)prob * n * n;
  const int c = blockIdx.x * TR_WARPS + warp;
  const int ctop = min(n, (blockIdx.x + 1) * TR_WARPS) - 1;   // highest column in this CTA

  cd y[QMAX];
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    const int r = lane + 32 * q;
    y[q] = (c < n && r <= c) ? cconj(V[c + (int64_t)r * m]) : cmk(0.0, 0.0);
  }
  if (c < n)   // panels wholly below row c stay zero
    for (int i = (c / nb + 1) * nb + lane; i < n; i += 32) M[i + (int64_t)c * n] = cmk(0.0, 0.0);

  auto stage = [&](int pi, int buf) {   // G[r, p0 + j], r < p0, j < pw
    if constexpr (!STAGE) return;
    const int p0 = pi * nb, pw = min(nb, n - p0);
    cd* dst = Gs + buf * nb * n;
    for (int e = threadIdx.x; e < pw * p0; e += blockDim.x) {
      const int r = e % p0, jj = e / p0;
      const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(dst + jj * n + r));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(G + r + (int64_t)(p0 + jj) * n));
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  const int pstart = ctop / nb;
  for (int e = threadIdx.x; STAGE && e < (pstart + 1) * nb * nb; e += blockDim.x) {   // T of panels 0 .. pstart
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(Ts + e));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(T + e));
  }
  stage(pstart, 0);   // the same commit group as T
  for (int pi = pstart; pi >= 0; --pi) {
    const int k = pstart - pi;
    if (pi > 0) {
      stage(pi - 1, (k + 1) & 1);
      if constexpr (STAGE) asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      if constexpr (STAGE) asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
    const int p0 = pi * nb, pw = min(nb, n - p0);
    if (c < n && p0 <= c) {   // warp-uniform
      const int qb = p0 >> 5, base = p0 & 31, ii = lane - base;   // the panel's rows sit in lanes base ..
      cd yb = cmk(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < QMAX; ++q)
        if (q == qb) yb = y[q];
      const cd* Tp = STAGE ? Ts + pi * nb * nb : T + (int64_t)pi * nb * nb;
      cd a0 = cmk(0.0, 0.0), a1 = cmk(0.0, 0.0);
      for (int jj = 0; jj < pw; ++jj) {
        const cd rj = cmk(__shfl_sync(0xffffffffu, yb.x, base + jj), __shfl_sync(0xffffffffu, yb.y, base + jj));
        if (ii >= 0 && ii <= jj) cfma((jj & 1) ? a1 : a0, Tp[ii + nb * jj], rj);
      }
      const cd mi = cadd(a0, a1);
      if (ii >= 0 && ii < pw) M[p0 + ii + (int64_t)c * n] = mi;
      const cd* Gc = Gs + (k & 1) * nb * n;
      for (int jj = 0; jj < pw; ++jj) {
        const cd mj = cmk(__shfl_sync(0xffffffffu, mi.x, base + jj), __shfl_sync(0xffffffffu, mi.y, base + jj));
        const cd* gcol = STAGE ? Gc + jj * n : G + (int64_t)(p0 + jj) * n;
#pragma unroll
        for (int q = 0; q < QMAX; ++q) {
          const int r = lane + 32 * q;
          if (r < p0) y[q] = csub(y[q], cmul(gcol[r], mj));
        }
      }
    }
    __syncthreads();   // this buffer is refilled by the next iteration's prefetch
  }
}

typedef void (*TmatKernel)(int, int, int, const cd*, const cd*, const cd*, cd*);

size_t tmat_smem(int n, int nb) { return (2 * (size_t)nb * n + (size_t)((n + nb - 1) / nb) * nb * nb) * sizeof(cd); }

// The staged variant when G's panel columns (double-buffered) and every T_p fit in shared
// memory, else the same algorithm reading them from global memory (L2).
template <bool ST>
TmatKernel tmat_pick(int n) {
  if (n <= 32) return qr_tmat_kernel<1, ST>;
  if (n <= 64) return qr_tmat_kernel<2, ST>;
  if (n <= 128) return qr_tmat_kernel<4, ST>;
  if (n <= 256) return qr_tmat_kernel<8, ST>;
  if (n <= 512) return qr_tmat_kernel<16, ST>;
  return nullptr;
}
TmatKernel tmat_kernel_for(int n, int nb) {
  return tmat_smem(n, nb) <= SMEM_LIMIT ? tmat_pick<true>(n) : tmat_pick<false>(n);
}

struct Choice {
  int C = 0, rpl = 0, nb = 0;
  size_t smem = 0;
};

// Cluster of C = ceil(m / (32 rpl)) CTAs, at most 16: prefer 1 row per lane (measured: the
// per-CTA work, not the exchange, sets the time), then 2, then 4; the widest panel that fits.
bool choose(int m, int n, Choice& ch) {
  QrParams P;
  for (int rpl : {1, 2, 4}) {
    const int rows = 32 * rpl;
    const int C = (m + rows - 1) / rows;
    if (C > CMAX) continue;
    for (int nb : {16, 8, 4}) {
      size_t b = layout(P, n, C, rows, nb);
      if (b <= SMEM_LIMIT) {
        ch.C = C; ch.rpl = rpl; ch.nb = nb; ch.smem = b;
        return true;
      }
    }
  }
  return false;
}

// Strided m x n matrix fill: COPY dst = src, UPPER dst = triu(src), IDENT dst = [I; 0].
enum { MAT_COPY = 0, MAT_UPPER, MAT_IDENT };
__global__ void mat_kernel(int mode, int m, int n, const cd* __restrict__ src, int64_t sr, int64_t sc, cd* dst,
                           int64_t dr, int64_t dc) {
  const int64_t total = (int64_t)m * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(e % m), k = (int)(e / m);
    cd v;
    if (mode == MAT_IDENT) v = cmk(g == k ? 1.0 : 0.0, 0.0);
    else if (mode == MAT_UPPER && k < g) v = cmk(0.0, 0.0);
    else v = src[g * sr + k * sc];
    dst[g * dr + k * dc] = v;
  }
}

int mat_launch(int mode, int m, int n, const cd* src, int64_t sr, int64_t sc, cd* dst, int64_t dr, int64_t dc,
               Workspace* ws, cudaStream_t s) {
  count_launch(ws);
  const int64_t total = (int64_t)m * n;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
  mat_kernel<<<blocks, 256, 0, s>>>(mode, m, n, src, sr, sc, dst, dr, dc);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

// The cluster factorisation of every problem of p: R (if requested), the explicit reflectors
// V [batch][n][m], the panels' T [batch][npanels][nb][nb], and E = [I; 0] in p.Q.
int launch_factor(const QrProblem& p, const Choice& ch, cd* Vb, cd* Tb, cudaStream_t s) {
  QrParams P;
  layout(P, p.n, ch.C, 32 * ch.rpl, ch.nb);
  P.p = p;
  P.V = Vb;
  P.Tg = Tb;
  QrKernel fn = kernel_for(ch.rpl, ch.nb);
  if (!fn) return MPSB_ERR_UNSUPPORTED;
  MPSB_TRY(ensure_kernel_attrs((const void*)fn, (int)SMEM_LIMIT, true));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ch.C, p.batch, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = ch.smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ch.C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MPSB_CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, P));
  return MPSB_OK;
}

// Q = E - V (T V1^H) for every problem of p, p.Q holding E: G = V^H V, the back substitution
// for M = T V1^H, and Q -= V M.
int form_q(const QrProblem& p, int nb, const cd* Vb, const cd* Tb, cd* Gb, cd* Mb, Workspace* ws, cudaStream_t s) {
  const int m = p.m, n = p.n;
  const TmatKernel tk = tmat_kernel_for(n, nb);
  if (!tk) return MPSB_ERR_UNSUPPORTED;
  const cd one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0), mone = cmk(-1.0, 0.0);
  {  // G = V^H V
    Gemm g;
    g.M = n; g.N = n; g.K = m; g.batch = p.batch;
    g.A = Vb; g.a_m = m; g.a_k = 1; g.a_b = (int64_t)m * n; g.conjA = true;
    g.B = Vb; g.b_k = 1; g.b_n = m; g.b_b = (int64_t)m * n;
    g.C = Gb; g.c_m = 1; g.c_n = n; g.c_b = (int64_t)n * n;
    g.alpha = one; g.beta = zero;
    MPSB_TRY(gemm_launch(g, ws, s));
  }
  {  // M = T V1^H
    const size_t smem = tmat_smem(n, nb) <= SMEM_LIMIT ? tmat_smem(n, nb) : 0;
    if (smem) MPSB_TRY(ensure_kernel_attrs((const void*)tk, (int)SMEM_LIMIT));
    count_launch(ws);
    tk<<<dim3((n + TR_WARPS - 1) / TR_WARPS, p.batch), 32 * TR_WARPS, smem, s>>>(m, n, nb, Vb, Tb, Gb, Mb);
    MPSB_CUDA_TRY(cudaGetLastError());
  }
  {  // Q = E - V M
    Gemm g;
    g.M = m; g.N = n; g.K = n; g.batch = p.batch;
    g.A = Vb; g.a_m = 1; g.a_k = m; g.a_b = (int64_t)m * n;
    g.B = Mb; g.b_k = 1; g.b_n = n; g.b_b = (int64_t)n * n;
    g.C = p.Q; g.c_m = p.q_r; g.c_n = p.q_c; g.c_b = p.q_b;
    g.alpha = mone; g.beta = one;
    MPSB_TRY(gemm_launch(g, ws, s));
  }
  return MPSB_OK;
}

// Blocked QR for one matrix beyond the cluster's shared memory (for example 2048 x 512): the
// working matrix is p.Q (X copied in unless they coincide); every 16-column panel is
// factored by the cluster kernel (its R rows written back in place, its reflectors and T
// kept), the trailing columns get A -= V (T^H (V^H A)) by three tensor-core GEMMs, and Q is
// formed from all reflectors as in the single-kernel path.
constexpr int BP = 16;

// The look-ahead lane of the blocked QR: created by the first (eager) call of a workspace.
int qr_side_lane(Workspace* ws) {
  if (ws->qr_side) return MPSB_OK;
  if (ws->capturing) {
    set_last_message("QR look-ahead lane first needed during graph capture");
    return MPSB_ERR_UNSUPPORTED;
  }
  MPSB_CUDA_TRY(cudaStreamCreateWithFlags(&ws->qr_side, cudaStreamNonBlocking));
  for (cudaEvent_t& e : ws->qr_ev) MPSB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  ws->qr_side_ws = new Workspace();
  return MPSB_OK;
}

// Right-looking blocked QR with look-ahead for shapes beyond one cluster (e.g. 2048 x 512):
// panels of BP columns, each factored by the cluster kernel.  Panel pi's block reflector
// I - V T V^H is applied to the next panel's columns on the main stream, which then factors
// that panel at once, while the same update of the columns after it runs on the look-ahead
// lane -- so the latency-bound panel factorisations overlap the trailing GEMMs.  Every column
// still gets the panels' updates in panel order (the main stream waits for the lane's update
// of panel pi-1 before it applies panel pi to the next panel), so the result is the
// unblocked order's.
int qr_blocked(const QrProblem& p, Workspace* ws, cudaStream_t s) {
  const int m = p.m, n = p.n, npan = (n + BP - 1) / BP;
  const int64_t qr_ = p.q_r, qc = p.q_c;
  // scratch: V [n][m], T [npan][16][16], G and M [n][n], panel V and E [16][m], W and W2 [n][16]
  // (the lane's trailing update), Wn and W2n [16][16] (the next panel's update)
  const size_t nV = (size_t)m * n, nT = (size_t)npan * BP * BP, nG = (size_t)n * n, nP = (size_t)m * BP,
               nW = (size_t)n * BP, nWn = (size_t)BP * BP;
  MPSB_TRY(devbuf_ensure(ws, ws->qr, (nV + nT + 2 * nG + 2 * nP + 2 * nW + 2 * nWn) * sizeof(cd)));
  MPSB_TRY(qr_side_lane(ws));
  Workspace* sw = ws->qr_side_ws;
  sw->capturing = ws->capturing;
  sw->per_problem = ws->per_problem;
  cudaStream_t ls = ws->qr_side;
  cudaEvent_t ev_v = ws->qr_ev[0], ev_t = ws->qr_ev[1];
  cd* Vb = static_cast<cd*>(ws->qr.p);
  cd* Tb = Vb + nV;
  cd* Gb = Tb + nT;
  cd* Mb = Gb + nG;
  cd* Vp = Mb + nG;
  cd* Ep = Vp + nP;
  cd* Wb = Ep + nP;
  cd* W2 = Wb + nW;
  cd* Wn = W2 + nW;
  cd* W2n = Wn + nWn;
  cd* A = p.Q;
  if (p.X != p.Q || p.x_r != qr_ || p.x_c != qc)
    MPSB_TRY(mat_launch(MAT_COPY, m, n, p.X, p.x_r, p.x_c, A, qr_, qc, ws, s));
  MPSB_CUDA_TRY(cudaMemsetAsync(Vb, 0, nV * sizeof(cd), s));
  const cd one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0), mone = cmk(-1.0, 0.0);

  // factor panel pi (its columns have every earlier panel's update) and keep its V in Vb
  auto factor = [&](int pi) -> int {
    const int p0 = pi * BP, pw = std::min(BP, n - p0), mp = m - p0;
    Choice ch;
    if (!choose(mp, pw, ch) || ch.nb != BP) {
      set_last_message("QR panel of %d x %d does not fit the cluster kernel", mp, pw);
      return MPSB_ERR_UNSUPPORTED;
    }
    cd* Ap = A + p0 * qr_ + p0 * qc;
    QrProblem pp;
    pp.m = mp; pp.n = pw; pp.batch = 1;
    pp.X = Ap; pp.x_r = qr_; pp.x_c = qc;
    pp.Q = Ep; pp.q_r = 1; pp.q_c = mp;
    pp.R = Ap; pp.r_r = qr_; pp.r_c = qc;   // R rows back in place (the panel's V is kept apart)
    pp.err = p.err;
    count_launch(ws);
    MPSB_TRY(launch_factor(pp, ch, Vp, Tb + (int64_t)pi * BP * BP, s));
    MPSB_CUDA_TRY(cudaMemcpy2DAsync(Vb + p0 + (int64_t)p0 * m, (size_t)m * sizeof(cd), Vp, (size_t)mp * sizeof(cd),
                                    (size_t)mp * sizeof(cd), pw, cudaMemcpyDeviceToDevice, s));
    return MPSB_OK;
  };
  // columns c0 .. c0 + nc - 1 of A <- (I - V T V^H)^H applied by panel pi, on stream st
  auto update = [&](int pi, int c0, int nc, cd* W, int ldw, cd* Wt, Workspace* w, cudaStream_t st) -> int {
    const int p0 = pi * BP, pw = std::min(BP, n - p0), mp = m - p0;
    const cd* V = Vb + p0 + (int64_t)p0 * m;   // rows p0.., leading dimension m
    cd* At = A + p0 * qr_ + (int64_t)c0 * qc;
    {  // W = V^H A_t
      Gemm g;
      g.M = pw; g.N = nc; g.K = mp;
      g.A = V; g.a_m = m; g.a_k = 1; g.conjA = true;
      g.B = At; g.b_k = qr_; g.b_n = qc;
      g.C = W; g.c_m = 1; g.c_n = ldw;
      g.alpha = one; g.beta = zero;
      MPSB_TRY(gemm_launch(g, w, st));
    }
    {  // Wt = T^H W
      Gemm g;
      g.M = pw; g.N = nc; g.K = pw;
      g.A = Tb + (int64_t)pi * BP * BP; g.a_m = BP; g.a_k = 1; g.conjA = true;
      g.B = W; g.b_k = 1; g.b_n = ldw;
      g.C = Wt; g.c_m = 1; g.c_n = ldw;
      g.alpha = one; g.beta = zero;
      MPSB_TRY(gemm_launch(g, w, st));
    }
    {  // A_t -= V Wt
      Gemm g;
      g.M = mp; g.N = nc; g.K = pw;
      g.A = V; g.a_m = 1; g.a_k = m;
      g.B = Wt; g.b_k = 1; g.b_n = ldw;
      g.C = At; g.c_m = qr_; g.c_n = qc;
      g.alpha = mone; g.beta = one;
      MPSB_TRY(gemm_launch(g, w, st));
    }
    return MPSB_OK;
  };

  MPSB_TRY(factor(0));
  bool lane_pending = false;   // the lane holds an update the main stream has not waited for
  for (int pi = 0; pi + 1 < npan; ++pi) {
    const int c1 = (pi + 1) * BP, nnext = std::min(BP, n - c1);
    const int c2 = c1 + nnext, nrest = n - c2;
    // the next panel's columns have panel pi-1's update only once the lane's update is done
    if (lane_pending) {
      MPSB_CUDA_TRY(cudaStreamWaitEvent(s, ev_t, 0));
      lane_pending = false;
    }
    int st = MPSB_OK;
    if (nrest > 0) {   // V_pi and T_pi are final on the main stream: fork the trailing update
      MPSB_CUDA_TRY(cudaEventRecord(ev_v, s));
      MPSB_CUDA_TRY(cudaStreamWaitEvent(ls, ev_v, 0));
      st = update(pi, c2, nrest, Wb, BP, W2, sw, ls);
      MPSB_CUDA_TRY(cudaEventRecord(ev_t, ls));   // recorded on failure too, so the join below holds
      lane_pending = true;
    }
    if (st == MPSB_OK) st = update(pi, c1, nnext, Wn, BP, W2n, ws, s);
    if (st == MPSB_OK) st = factor(pi + 1);
    if (st != MPSB_OK) {   // never leave the lane forked
      cudaStreamWaitEvent(s, ev_t, 0);
      return st;
    }
  }
  if (lane_pending) MPSB_CUDA_TRY(cudaStreamWaitEvent(s, ev_t, 0));   // join the lane
  ws->launches += sw->launches;
  sw->launches = 0;
  if (p.R) MPSB_TRY(mat_launch(MAT_UPPER, n, n, A, qr_, qc, p.R, p.r_r, p.r_c, ws, s));
  MPSB_TRY(mat_launch(MAT_IDENT, m, n, nullptr, 0, 0, A, qr_, qc, ws, s));
  QrProblem q = p;
  return form_q(q, BP, Vb, Tb, Gb, Mb, ws, s);
}

bool blocked_ok(int m, int n) {
  Choice ch;
  return n <= 512 && choose(m, std::min(n, BP), ch) && ch.nb == BP;
}

}  // namespace

bool qr_batch_supported(int m, int n) {
  Choice ch;
  return m >= n && n >= 1 && n <= 512 && choose(m, n, ch);
}

bool qr_supported(int m, int n) {
  Choice ch;
  return m >= n && n >= 1 && n <= 512 && (choose(m, n, ch) || blocked_ok(m, n));
}

int qr_launch(const QrProblem& p, Workspace* ws, cudaStream_t s) {
  if (p.m < p.n || p.n < 1 || p.batch < 1) return MPSB_ERR_DIMENSION;
  if (p.batch > 65535) return MPSB_ERR_UNSUPPORTED;
  if (!ws) return MPSB_ERR_INVALID_ARG;
  const int m = p.m, n = p.n;
  Choice ch;
  if (n > 512 || (!choose(m, n, ch) && (p.batch != 1 || !blocked_ok(m, n)))) {
    set_last_message("QR of a %d x %d matrix (batch %d) is beyond the supported shapes", m, n, p.batch);
    return MPSB_ERR_UNSUPPORTED;
  }
  if (!choose(m, n, ch)) return qr_blocked(p, ws, s);
  const int nb = ch.nb, npan = (n + nb - 1) / nb;
  // scratch: V [batch][n][m], the panels' T [batch][npan][nb][nb], G = V^H V and
  // M = T V1^H [batch][n][n] each
  const size_t nV = (size_t)p.batch * m * n, nT = (size_t)p.batch * npan * nb * nb, nG = (size_t)p.batch * n * n;
  MPSB_TRY(devbuf_ensure(ws, ws->qr, (nV + nT + 2 * nG) * sizeof(cd)));
  cd* Vb = static_cast<cd*>(ws->qr.p);
  cd* Tb = Vb + nV;
  cd* Gb = Tb + nT;
  cd* Mb = Gb + nG;
  MPSB_TRY(launch_factor(p, ch, Vb, Tb, s));
  return form_q(p, nb, Vb, Tb, Gb, Mb, ws, s);
}

}  // namespace mpsb
