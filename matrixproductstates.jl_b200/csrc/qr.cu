// Householder QR with the LAPACK zgeqrf + zungqr conventions (the routines qrq! calls,
// src/orthonormalisation.jl:180-184), Q (and optionally R) of an m x n complex matrix, m >= n.
//
// Reflector convention (zlarfg): for column j with alpha = A[j,j] and x = A[j+1:m, j],
//   if x == 0 and Im(alpha) == 0:  tau = 0 (H = I, R[j,j] = alpha)
//   else beta = -copysign(|(alpha, x)|, Re alpha), tau = (beta - alpha)/beta,
//        v = [1; x/(alpha - beta)], R[j,j] = beta (real)
// H(j)^H = I - conj(tau) v v^H is applied to the trailing columns (zgeqr2), and
// Q = H(1)...H(n) [I; 0] (zungqr).  Because only the span of Q carries physics in the
// sweeps, the one convention that must match LAPACK exactly is the sign / phase rule
// above, which also fixes the "junk" columns of zero-padded (rank-deficient) sites.
//
// B200 mapping: one thread-block cluster per matrix; the m rows are split over the C
// CTAs of the cluster (ROWS rows each, the whole matrix lives in distributed shared
// memory).  Blocked right-looking algorithm with panels of nb columns:
//   * panel column j: every CTA reduces its rows (norm, dot products with the remaining
//     panel columns, and V^H x for the compact-WY factor T), one cluster barrier, every
//     CTA gathers the C partial sets over DSMEM in a fixed order (so all CTAs compute
//     bit-identical reflectors) and updates its rows;
//   * trailing columns: W = V^H A partials -> barrier -> reduce-scatter + T^H ->
//     barrier -> all-gather -> A -= V W (two barriers per panel);
//   * Q formation runs the panels backwards with Q_trail -= V (T (V^H Q_trail)) and the
//     panel block built directly as E - V (T V1^H) (two barriers per panel).
// All reductions are in a fixed order: results are reproducible run to run.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace mpsb {
namespace {

constexpr int NT = 256;
constexpr size_t SMEM_LIMIT = 227 * 1024;

struct QrParams {
  QrProblem p;
  int C, rows, nb, npanels, ldS;
  // shared-memory offsets (in complex elements)
  int o_S, o_step, o_bc, o_wpart, o_w2s, o_T, o_v1pub, o_v1loc, o_mloc, o_red;
  int step_elems, w2s_cols;
};

// ---- per-CTA shared memory map ------------------------------------------------------
// S      [(rows+1) * n]   local rows of the matrix, column-major, ld = rows+1
// step   2 x [2*nb]       pq[nb] (partial dot products), rowj[nb] (published row j)
// bc     [4 + 4*nb]       tau, beta, scale, pad, w[nb], t[nb], sumpq[nb], rowjl[nb]
// wpart  [nb * n]         trailing partials V^H A (this CTA's rows); reused as the gathered W2
// w2s    [nb * w2s_cols]  this CTA's reduced slice of W2
// T      [npanels*nb*nb]  compact-WY triangular factors of all panels
// v1pub / v1loc / mloc [nb*nb]  panel-top block of V (published / gathered), M = T V1^H
// red    [NT/32]          cross-warp reduction scratch

template <int ROWS>
__device__ __forceinline__ cd group_sum(cd v, cd* red) {
  constexpr int W = ROWS < 32 ? ROWS : 32;
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
  }
  if constexpr (ROWS <= 32) {
    return v;
  } else {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    cd s = cmk(0.0, 0.0);
    if (tid % ROWS == 0) {
#pragma unroll
      for (int w = 0; w < ROWS / 32; ++w) s = cadd(s, red[warp + w]);
    }
    return s;
  }
}

template <int ROWS>
__global__ void __launch_bounds__(NT, 1) qr_kernel(QrParams P) {
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* sm = reinterpret_cast<cd*>(smem_raw);
  constexpr int G = NT / ROWS;   // column groups
  const int C = P.C, nb = P.nb, ldS = P.ldS;
  const int m = P.p.m, n = P.p.n;
  const int crank = (int)cluster.block_rank();
  const int prob = blockIdx.y;
  const int tid = threadIdx.x;
  const int r = tid % ROWS, grp = tid / ROWS;
  const int row0 = crank * ROWS;
  const int grow = row0 + r;

  cd* S = sm + P.o_S;
  cd* bc = sm + P.o_bc;
  cd* bw = bc + 4;          // w[nb]
  cd* bt = bw + nb;         // t[nb]
  cd* sumpq = bt + nb;      // [nb]
  cd* rowjl = sumpq + nb;   // [nb]
  cd* wpart = sm + P.o_wpart;
  cd* w2s = sm + P.o_w2s;
  cd* Tall = sm + P.o_T;
  cd* v1pub = sm + P.o_v1pub;
  cd* v1loc = sm + P.o_v1loc;
  cd* mloc = sm + P.o_mloc;
  cd* red = sm + P.o_red;

  // ---- load this CTA's rows
  {
    const cd* X = P.p.X + (int64_t)prob * P.p.x_b;
    for (int e = tid; e < ROWS * n; e += NT) {
      int rr = e % ROWS, cc = e / ROWS, g = row0 + rr;
      S[cc * ldS + rr] = (g < m) ? X[(int64_t)g * P.p.x_r + (int64_t)cc * P.p.x_c] : cmk(0.0, 0.0);
    }
  }
  cluster.sync();

  // ================================ factorisation ================================
  int sp = 0;
  for (int pi = 0; pi < P.npanels; ++pi) {
    const int p0 = pi * nb;
    const int pw = min(nb, n - p0);
    cd* Tp = Tall + pi * nb * nb;
    for (int jl = 0; jl < pw; ++jl) {
      const int j = p0 + jl;
      cd* st = sm + P.o_step + sp * P.step_elems;   // pq[nb], rowj[nb]
      // -- phase A: partial sums over this CTA's rows g > j
      {
        cd x = cmk(0.0, 0.0);
        if (grow > j && grow < m) x = S[j * ldS + r];
        const int nslots = (pw + G - 1) / G;
        for (int s = 0; s < nslots; ++s) {
          int c = grp + G * s;
          cd v = cmk(0.0, 0.0);
          if (c < pw && grow > j && grow < m) {
            cd a = S[(p0 + c) * ldS + r];
            if (c >= jl) { v = cmul(cconj(x), a); }
            else         { v = cmul(cconj(a), x); }
          }
          v = group_sum<ROWS>(v, red);
          if (r == 0 && c < pw) st[c] = v;
        }
        if (j >= row0 && j < row0 + ROWS && tid < pw) st[nb + tid] = S[(p0 + tid) * ldS + (j - row0)];
      }
      cluster.sync();
      // -- phase B: gather (fixed order), reflector, w / t, T column
      if (tid < pw) {
        cd s = cmk(0.0, 0.0);
        for (int q = 0; q < C; ++q) s = cadd(s, cluster.map_shared_rank(st, q)[tid]);
        sumpq[tid] = s;
      } else if (tid >= 64 && tid < 64 + pw) {
        int c = tid - 64;
        rowjl[c] = cluster.map_shared_rank(st, j / ROWS)[nb + c];
      }
      __syncthreads();
      if (tid == 0) {
        cd alpha = rowjl[jl];
        double xn2 = sumpq[jl].x;
        cd tau, beta, scale;
        if (xn2 == 0.0 && alpha.y == 0.0) {
          tau = cmk(0.0, 0.0); beta = alpha; scale = cmk(1.0, 0.0);
        } else {
          double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
          double b = -copysign(nrm, alpha.x);
          tau = cmk((b - alpha.x) / b, -alpha.y / b);
          beta = cmk(b, 0.0);
          scale = crecip(cmk(alpha.x - b, alpha.y));
        }
        bc[0] = tau; bc[1] = beta; bc[2] = scale;
      }
      __syncthreads();
      const cd tau = bc[0], beta = bc[1], scale = bc[2];
      if (tid < pw) {
        int c = tid;
        if (c > jl) bw[c] = cadd(rowjl[c], cmul(cconj(scale), sumpq[c]));
        else if (c < jl) bt[c] = cadd(cconj(rowjl[c]), cmul(scale, sumpq[c]));
      }
      // v for this thread's row (read before the column is rewritten)
      cd vr = cmk(0.0, 0.0);
      if (grow == j) vr = cmk(1.0, 0.0);
      else if (grow > j && grow < m) vr = cmul(scale, S[j * ldS + r]);
      __syncthreads();
      // T column jl:  T[i, jl] = -tau * sum_{i'=i}^{jl-1} T[i, i'] t[i'],  T[jl, jl] = tau
      if (tid < jl) {
        cd s = cmk(0.0, 0.0);
        for (int i2 = tid; i2 < jl; ++i2) cfma(s, Tp[tid + nb * i2], bt[i2]);
        Tp[tid + nb * jl] = cmul(cmk(-tau.x, -tau.y), s);
      } else if (tid == jl) {
        Tp[jl + nb * jl] = tau;
      }
      const bool active = (tau.x != 0.0) || (tau.y != 0.0);
      if (active) {
        if (grp == 0) {
          if (grow == j) S[j * ldS + r] = beta;
          else if (grow > j && grow < m) S[j * ldS + r] = vr;
        }
        if (grow >= j && grow < m) {
          const cd ctv = cmul(cconj(tau), vr);
          for (int c = jl + 1 + grp; c < pw; c += G) {
            cd* a = &S[(p0 + c) * ldS + r];
            *a = csub(*a, cmul(ctv, bw[c]));
          }
        }
      }
      __syncthreads();
      sp ^= 1;
    }

    // -- trailing update A_t := (I - V T^H V^H) A_t
    const int nt = n - p0 - pw;
    if (nt > 0) {
      const int kb = p0 + pw;
      for (int e = tid; e < pw * nt; e += NT) {
        int k = e % nt, i = e / nt;
        cd acc = cmk(0.0, 0.0);
        const int lo = max(0, p0 + i - row0);
        const int hi = min(ROWS, m - row0);
        for (int rr = lo; rr < hi; ++rr) {
          cd v = (row0 + rr == p0 + i) ? cmk(1.0, 0.0) : S[(p0 + i) * ldS + rr];
          cfma_cj(acc, v, S[(kb + k) * ldS + rr]);
        }
        wpart[i + nb * k] = acc;
      }
      cluster.sync();
      const int KS = (nt + C - 1) / C;
      const int k0 = crank * KS, k1 = min(nt, k0 + KS);
      for (int e = tid; e < pw * max(0, k1 - k0); e += NT) {
        int i = e % pw, k = k0 + e / pw;
        cd s = cmk(0.0, 0.0);
        for (int q = 0; q < C; ++q) s = cadd(s, cluster.map_shared_rank(wpart, q)[i + nb * k]);
        w2s[i + nb * (k - k0)] = s;
      }
      __syncthreads();
      // W2 = T^H W, column by column, descending i in place
      for (int k = k0 + tid; k < k1; k += NT) {
        cd* wcol = w2s + nb * (k - k0);
        for (int i = pw - 1; i >= 0; --i) {
          cd s = cmk(0.0, 0.0);
          for (int i2 = 0; i2 <= i; ++i2) cfma_cj(s, Tp[i2 + nb * i], wcol[i2]);
          wcol[i] = s;
        }
      }
      cluster.sync();
      for (int e = tid; e < pw * nt; e += NT) {
        int i = e % pw, k = e / pw, q = k / KS;
        wpart[i + nb * k] = cluster.map_shared_rank(w2s, q)[i + nb * (k - q * KS)];
      }
      __syncthreads();
      for (int e = tid; e < ROWS * nt; e += NT) {
        int rr = e % ROWS, k = e / ROWS;
        int g = row0 + rr;
        if (g < p0 || g >= m) continue;
        cd acc = cmk(0.0, 0.0);
        const int imax = min(pw - 1, g - p0);
        for (int i = 0; i <= imax; ++i) {
          cd v = (g == p0 + i) ? cmk(1.0, 0.0) : S[(p0 + i) * ldS + rr];
          cfma(acc, v, wpart[i + nb * k]);
        }
        cd* a = &S[(kb + k) * ldS + rr];
        *a = csub(*a, acc);
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
  // rows above each column's panel start are zero in the partially formed Q
  for (int e = tid; e < ROWS * n; e += NT) {
    int rr = e % ROWS, k = e / ROWS, g = row0 + rr;
    if (g < (k / nb) * nb) S[k * ldS + rr] = cmk(0.0, 0.0);
  }
  __syncthreads();

  // ================================ Q formation ==================================
  for (int pi = P.npanels - 1; pi >= 0; --pi) {
    const int p0 = pi * nb;
    const int pw = min(nb, n - p0);
    const int nt = n - p0 - pw, kb = p0 + pw;
    const cd* Tp = Tall + pi * nb * nb;
    // partials V^H Q_trail and the published top block V1[c, i] = V[p0 + c, i]
    for (int e = tid; e < pw * nt; e += NT) {
      int k = e % nt, i = e / nt;
      cd acc = cmk(0.0, 0.0);
      const int lo = max(0, p0 + i - row0);
      const int hi = min(ROWS, m - row0);
      for (int rr = lo; rr < hi; ++rr) {
        cd v = (row0 + rr == p0 + i) ? cmk(1.0, 0.0) : S[(p0 + i) * ldS + rr];
        cfma_cj(acc, v, S[(kb + k) * ldS + rr]);
      }
      wpart[i + nb * k] = acc;
    }
    for (int e = tid; e < pw * pw; e += NT) {
      int c = e % pw, i = e / pw, g = p0 + c;
      if (g >= row0 && g < row0 + ROWS) {
        cd v = (c == i) ? cmk(1.0, 0.0) : (c > i ? S[(p0 + i) * ldS + (g - row0)] : cmk(0.0, 0.0));
        v1pub[c + nb * i] = v;
      }
    }
    cluster.sync();
    const int KS = (nt + C - 1) / C;
    const int k0 = crank * KS, k1 = min(nt, k0 + KS);
    for (int e = tid; e < pw * max(0, k1 - k0); e += NT) {
      int i = e % pw, k = k0 + e / pw;
      cd s = cmk(0.0, 0.0);
      for (int q = 0; q < C; ++q) s = cadd(s, cluster.map_shared_rank(wpart, q)[i + nb * k]);
      w2s[i + nb * (k - k0)] = s;
    }
    for (int e = tid; e < pw * pw; e += NT) {
      int c = e % pw, i = e / pw;
      v1loc[c + nb * i] = cluster.map_shared_rank(v1pub, (p0 + c) / ROWS)[c + nb * i];
    }
    __syncthreads();
    // W2 = T W, ascending i in place
    for (int k = k0 + tid; k < k1; k += NT) {
      cd* wcol = w2s + nb * (k - k0);
      for (int i = 0; i < pw; ++i) {
        cd s = cmk(0.0, 0.0);
        for (int i2 = i; i2 < pw; ++i2) cfma(s, Tp[i + nb * i2], wcol[i2]);
        wcol[i] = s;
      }
    }
    // M = T V1^H  (M[i, c] = sum_{i2 >= i} T[i, i2] conj(V1[c, i2]))
    for (int e = tid; e < pw * pw; e += NT) {
      int i = e % pw, c = e / pw;
      cd s = cmk(0.0, 0.0);
      for (int i2 = i; i2 <= c && i2 < pw; ++i2) cfma(s, Tp[i + nb * i2], cconj(v1loc[c + nb * i2]));
      mloc[i + nb * c] = s;
    }
    cluster.sync();
    for (int e = tid; e < pw * nt; e += NT) {
      int i = e % pw, k = e / pw, q = k / KS;
      wpart[i + nb * k] = cluster.map_shared_rank(w2s, q)[i + nb * (k - q * KS)];
    }
    __syncthreads();
    // Q_trail -= V W2
    for (int e = tid; e < ROWS * nt; e += NT) {
      int rr = e % ROWS, k = e / ROWS, g = row0 + rr;
      if (g < p0 || g >= m) continue;
      cd acc = cmk(0.0, 0.0);
      const int imax = min(pw - 1, g - p0);
      for (int i = 0; i <= imax; ++i) {
        cd v = (g == p0 + i) ? cmk(1.0, 0.0) : S[(p0 + i) * ldS + rr];
        cfma(acc, v, wpart[i + nb * k]);
      }
      cd* a = &S[(kb + k) * ldS + rr];
      *a = csub(*a, acc);
    }
    __syncthreads();
    // panel block: Q[g, p0 + c] = delta(g, p0 + c) - sum_i V[g, i] M[i, c]
    cd qv[(NT / 8 + 1)];   // upper bound on columns per thread (pw / G + 1 <= 33)
    int cnt = 0;
    const int g = grow;
    for (int c = grp; c < pw; c += G) {
      cd acc = cmk(0.0, 0.0);
      if (g >= p0 && g < m) {
        const int imax = min(pw - 1, g - p0);
        for (int i = 0; i <= imax; ++i) {
          cd v = (g == p0 + i) ? cmk(1.0, 0.0) : S[(p0 + i) * ldS + r];
          cfma(acc, v, mloc[i + nb * c]);
        }
      }
      cd d = (g == p0 + c) ? cmk(1.0, 0.0) : cmk(0.0, 0.0);
      qv[cnt++] = csub(d, acc);
    }
    __syncthreads();
    cnt = 0;
    for (int c = grp; c < pw; c += G) S[(p0 + c) * ldS + r] = qv[cnt++];
    __syncthreads();
  }

  // ---- write Q (this CTA's rows)
  {
    cd* Q = P.p.Q + (int64_t)prob * P.p.q_b;
    for (int e = tid; e < ROWS * n; e += NT) {
      int rr = e % ROWS, cc = e / ROWS, g = row0 + rr;
      if (g < m) Q[(int64_t)g * P.p.q_r + (int64_t)cc * P.p.q_c] = S[cc * ldS + rr];
    }
  }
  // keep this CTA's shared memory alive until every peer has finished its DSMEM reads
  cluster.sync();
}

typedef void (*QrKernel)(QrParams);

QrKernel kernel_for(int rows) {
  switch (rows) {
    case 8: return qr_kernel<8>;
    case 16: return qr_kernel<16>;
    case 32: return qr_kernel<32>;
    case 64: return qr_kernel<64>;
    case 128: return qr_kernel<128>;
    case 256: return qr_kernel<256>;
    default: return nullptr;
  }
}

int next_pow2(int v) {
  int p = 8;
  while (p < v) p <<= 1;
  return p;
}

size_t layout(QrParams& P, int m, int n, int C, int rows, int nb) {
  P.C = C; P.rows = rows; P.nb = nb;
  P.npanels = (n + nb - 1) / nb;
  P.ldS = rows + 1;
  P.step_elems = 2 * nb;
  P.w2s_cols = (n + C - 1) / C;
  int o = 0;
  P.o_S = o;      o += P.ldS * n;
  P.o_step = o;   o += 2 * P.step_elems;
  P.o_bc = o;     o += 4 + 4 * nb;
  P.o_wpart = o;  o += nb * n;
  P.o_w2s = o;    o += nb * P.w2s_cols;
  P.o_T = o;      o += P.npanels * nb * nb;
  P.o_v1pub = o;  o += nb * nb;
  P.o_v1loc = o;  o += nb * nb;
  P.o_mloc = o;   o += nb * nb;
  P.o_red = o;    o += NT / 32;
  (void)m;
  return (size_t)o * sizeof(cd);
}

// Pick (cluster size, rows per CTA, panel width): the smallest cluster whose CTAs hold at
// most 64 rows (fewer barriers per column vs. more rows per CTA), then the widest panel that
// fits in shared memory.  MPSB_QR_CLUSTER overrides the cluster size (tuning).
bool choose(int m, int n, QrParams& P, size_t& smem) {
  static const int env_c = [] {
    const char* s = getenv("MPSB_QR_CLUSTER");
    return s ? atoi(s) : 0;
  }();
  const int cands[] = {1, 2, 4, 8, 16};
  for (int pass = 0; pass < 2; ++pass) {
    for (int C : cands) {
      if (env_c > 0 && C != env_c) continue;
      int rows = next_pow2((m + C - 1) / C);
      if (rows > 256) continue;
      if (pass == 0 && rows > 64 && C < 16 && env_c == 0) continue;
      for (int nb : {32, 16, 8, 4}) {
        if (nb > n && nb > 4) continue;
        size_t b = layout(P, m, n, C, rows, nb);
        if (b <= SMEM_LIMIT) { smem = b; return true; }
      }
    }
  }
  return false;
}

}  // namespace

bool qr_supported(int m, int n) {
  QrParams P;
  size_t smem;
  return m >= n && n >= 1 && choose(m, n, P, smem);
}

int qr_launch(const QrProblem& p, cudaStream_t s) {
  if (p.m < p.n || p.n < 1 || p.batch < 1) return MPSB_ERR_DIMENSION;
  if (p.batch > 65535) return MPSB_ERR_UNSUPPORTED;
  QrParams P;
  size_t smem;
  if (!choose(p.m, p.n, P, smem)) {
    set_last_message("QR of a %d x %d matrix exceeds the cluster shared-memory capacity", p.m, p.n);
    return MPSB_ERR_UNSUPPORTED;
  }
  P.p = p;
  QrKernel fn = kernel_for(P.rows);
  if (!fn) return MPSB_ERR_UNSUPPORTED;
  static bool attr_done[9] = {false};
  int key = 0;
  while ((8 << key) < P.rows) ++key;
  if (!attr_done[key]) {
    MPSB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_LIMIT));
    MPSB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    attr_done[key] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P.C, p.batch, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = P.C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MPSB_CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, P));
  return MPSB_OK;
}

}  // namespace mpsb
