// Thin SVD of a complex m x n matrix (FP64) by one-sided (Hestenes) Jacobi, for the truncation
// rule of compressionSVD! (src/compression.jl:1280-1312), whose `svd` is LAPACK's.
//
// The columns of W = X (or X^H when m < n, then U and V swap roles) are rotated pairwise until
// mutually orthogonal; V accumulates the rotations, the singular values are the final column
// norms, U the normalised columns.  For a pair (p, q) with alpha = |w_p|^2, beta = |w_q|^2,
// gamma = w_p^H w_q = |gamma| e^{i phi}: with b = e^{-i phi} w_q the 2x2 Gram matrix is real,
// zeta = (beta - alpha) / (2 |gamma|), t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)),
// c = 1 / sqrt(1 + t^2), s = c t, and w_p <- c w_p - s b, w_q <- s w_p + c b (likewise V).
// Relative accuracy of one-sided Jacobi holds for the small singular values as well, which the
// cumulative-weight cut of the truncation rule relies on.
//
// B200 mapping: one cooperative launch per matrix; CTA b takes pair b of each round of the
// round-robin tournament (n_pad / 2 disjoint pairs per round, n_pad - 1 rounds per sweep),
// reduces the three inner products over the rows with warp shuffles, rotates its two columns
// of W and V, and the grid barrier separates rounds.  A sweep in which no pair needed a
// rotation ends the loop; at most SVD_MAX_SWEEPS sweeps run (the kernel always finishes).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "workspace.cuh"

namespace cg = cooperative_groups;

namespace mpsb {
namespace {

constexpr int SVD_NT = 256, SVD_MAX_SWEEPS = 60;

__device__ __forceinline__ cd block_sum(cd v, cd* red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  cd s = cmk(0.0, 0.0);
  for (int w = 0; w < SVD_NT / 32; ++w) s = cadd(s, red[w]);   // fixed order: reproducible
  return s;
}

// partner of slot i in round r of the circle method over np (even) players: player 0 fixed
__device__ __forceinline__ void round_pair(int r, int b, int np, int& p, int& q) {
  const int m = np - 1;
  auto pos = [&](int slot) { return slot == 0 ? 0 : 1 + (slot - 1 + r) % m; };
  p = pos(b);
  q = pos(np - 1 - b);
  if (p > q) { const int t = p; p = q; q = t; }
}

__global__ void __launch_bounds__(SVD_NT) jacobi_kernel(int m, int np, cd* W, cd* V, int* flags, double eps) {
  cg::grid_group grid = cg::this_grid();
  __shared__ cd red[SVD_NT / 32];
  __shared__ int s_rot;
  const int b = blockIdx.x;
  for (int sweep = 0; sweep < SVD_MAX_SWEEPS; ++sweep) {
    for (int r = 0; r < np - 1; ++r) {
      int p, q;
      round_pair(r, b, np, p, q);
      cd* wp = W + (int64_t)p * m;
      cd* wq = W + (int64_t)q * m;
      cd a = cmk(0.0, 0.0), g = cmk(0.0, 0.0);
      double bb = 0.0;
      for (int i = threadIdx.x; i < m; i += SVD_NT) {
        const cd x = wp[i], y = wq[i];
        a.x += x.x * x.x + x.y * x.y;
        bb += y.x * y.x + y.y * y.y;
        cfma_cj(g, x, y);
      }
      a.y = bb;
      const cd ab = block_sum(a, red);
      const cd gm = block_sum(g, red);
      const double alpha = ab.x, beta = ab.y, ag = sqrt(gm.x * gm.x + gm.y * gm.y);
      if (ag > eps * sqrt(alpha * beta) && ag > 0.0) {
        const double zeta = (beta - alpha) / (2.0 * ag);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        const cd ph = cmk(gm.x / ag, -gm.y / ag);   // e^{-i phi}
        for (int i = threadIdx.x; i < m; i += SVD_NT) {
          const cd x = wp[i], y = cmul(ph, wq[i]);
          wp[i] = cmk(c * x.x - s * y.x, c * x.y - s * y.y);
          wq[i] = cmk(s * x.x + c * y.x, s * x.y + c * y.y);
        }
        cd* vp = V + (int64_t)p * np;
        cd* vq = V + (int64_t)q * np;
        for (int i = threadIdx.x; i < np; i += SVD_NT) {
          const cd x = vp[i], y = cmul(ph, vq[i]);
          vp[i] = cmk(c * x.x - s * y.x, c * x.y - s * y.y);
          vq[i] = cmk(s * x.x + c * y.x, s * x.y + c * y.y);
        }
        if (threadIdx.x == 0) atomicOr(&flags[sweep], 1);
      }
      grid.sync();
    }
    if (threadIdx.x == 0) s_rot = atomicAdd(&flags[sweep], 0);
    __syncthreads();
    if (s_rot == 0) break;   // every CTA reads the same final flag of this sweep
    grid.sync();
  }
}

// W <- op(X) (X^H when `adj`), padded with a zero column to even width; V <- I
__global__ void svd_init_kernel(int m, int n, int np, const cd* X, int64_t xr, int64_t xc, bool adj, cd* W, cd* V) {
  const int64_t tw = (int64_t)m * np, tv = (int64_t)np * np;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tw + tv; e += (int64_t)gridDim.x * blockDim.x) {
    if (e < tw) {
      const int i = (int)(e % m), j = (int)(e / m);
      cd v = cmk(0.0, 0.0);
      if (j < n) v = adj ? cconj(X[(int64_t)j * xr + (int64_t)i * xc]) : X[(int64_t)i * xr + (int64_t)j * xc];
      W[e] = v;
    } else {
      const int64_t f = e - tw;
      V[f] = cmk((f % np) == (f / np) ? 1.0 : 0.0, 0.0);
    }
  }
}

__global__ void col_norms_kernel(int m, int np, const cd* W, double* s) {
  __shared__ cd red[SVD_NT / 32];
  const cd* w = W + (int64_t)blockIdx.x * m;
  cd a = cmk(0.0, 0.0);
  for (int i = threadIdx.x; i < m; i += SVD_NT) a.x += w[i].x * w[i].x + w[i].y * w[i].y;
  a = block_sum(a, red);
  if (threadIdx.x == 0) s[blockIdx.x] = sqrt(a.x);
}

// sorted outputs: Lout[:, k] = W[:, perm[k]] / s (left vectors of op(X)), Rout[:, k] = V[:, perm[k]]
__global__ void svd_gather_kernel(int m, int np, int k, const cd* W, const cd* V, const double* s, const int* perm,
                                  cd* Lout, int64_t l_r, int64_t l_c, cd* Rout, int64_t r_r, int64_t r_c, int nr) {
  const int64_t tl = (int64_t)m * k, tr = (int64_t)nr * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tl + tr; e += (int64_t)gridDim.x * blockDim.x) {
    if (e < tl) {
      const int i = (int)(e % m), j = (int)(e / m), c = perm[j];
      const double sv = s[c];
      const cd w = W[(int64_t)c * m + i];
      Lout[i * l_r + (int64_t)j * l_c] = sv > 0 ? cmk(w.x / sv, w.y / sv) : cmk(0.0, 0.0);
    } else {
      const int64_t f = e - tl;
      const int i = (int)(f % nr), j = (int)(f / nr);
      Rout[i * r_r + (int64_t)j * r_c] = V[(int64_t)perm[j] * np + i];
    }
  }
}

}  // namespace

// Thin SVD X = U diag(S) V^H (m x n, k = min(m, n) singular values, descending, S on the host
// and in `dS` if non-null).  U: m x k with strides (u_r, u_c); V: n x k with (v_r, v_c).
int svd_launch(int m, int n, const cd* X, int64_t x_r, int64_t x_c, cd* U, int64_t u_r, int64_t u_c, double* S,
               cd* V, int64_t v_r, int64_t v_c, Workspace* ws, cudaStream_t st) {
  if (m < 1 || n < 1) return MPSB_ERR_DIMENSION;
  const bool adj = m < n;
  const int mm = adj ? n : m, nn = adj ? m : n, np = nn + (nn & 1), k = nn;
  if (np / 2 > 1024) return MPSB_ERR_UNSUPPORTED;
  const size_t bytes = ((size_t)mm * np + (size_t)np * np) * sizeof(cd) + np * sizeof(double) + np * sizeof(int) +
                       SVD_MAX_SWEEPS * sizeof(int) + 64;
  MPSB_TRY(devbuf_ensure(ws, ws->svd, bytes));
  cd* W = static_cast<cd*>(ws->svd.p);
  cd* Vw = W + (int64_t)mm * np;
  double* dS = reinterpret_cast<double*>(Vw + (int64_t)np * np);
  int* dperm = reinterpret_cast<int*>(dS + np);
  int* flags = dperm + np;
  MPSB_CUDA_TRY(cudaMemsetAsync(flags, 0, SVD_MAX_SWEEPS * sizeof(int), st));
  count_launch(ws);
  svd_init_kernel<<<148 * 4, 256, 0, st>>>(mm, nn, np, X, x_r, x_c, adj, W, Vw);
  MPSB_CUDA_TRY(cudaGetLastError());
  if (np >= 2) {
    int nb = np / 2;
    int mmv = mm;
    double eps = 1e-15;
    void* args[] = {&mmv, (void*)&np, &W, &Vw, &flags, &eps};
    count_launch(ws);
    MPSB_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)jacobi_kernel, dim3(nb), dim3(SVD_NT), args, 0, st));
  }
  count_launch(ws);
  col_norms_kernel<<<np, SVD_NT, 0, st>>>(mm, np, W, dS);
  MPSB_CUDA_TRY(cudaGetLastError());
  std::vector<double> hs(np);
  MPSB_CUDA_TRY(cudaMemcpyAsync(hs.data(), dS, np * sizeof(double), cudaMemcpyDeviceToHost, st));
  MPSB_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<int> perm(np);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.begin() + np, [&](int a, int b) { return hs[a] > hs[b]; });
  // the padding column (zero) sorts last; keep the k largest
  for (int j = 0; j < k; ++j) S[j] = hs[perm[j]];
  MPSB_CUDA_TRY(cudaMemcpyAsync(dperm, perm.data(), np * sizeof(int), cudaMemcpyHostToDevice, st));
  count_launch(ws);
  // op(X) = L S R^H with L = normalised W, R = V: for X itself U = L, V = R; for X^H, U = R, V = L
  if (!adj)
    svd_gather_kernel<<<148 * 4, 256, 0, st>>>(mm, np, k, W, Vw, dS, dperm, U, u_r, u_c, V, v_r, v_c, nn);
  else
    svd_gather_kernel<<<148 * 4, 256, 0, st>>>(mm, np, k, W, Vw, dS, dperm, V, v_r, v_c, U, u_r, u_c, nn);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

}  // namespace mpsb

// ---- compressionSVD! (src/compression.jl:1280-1312) -------------------------------------
#include "engine.cuh"

namespace mpsb {
namespace {

// out (rows x cols, ld rows) = the conjugate transpose of the first `rows` columns of V (cols x rows used)
__global__ void adjoint_cols_kernel(int rows, int cols, const cd* V, int64_t ldv, cd* out) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(e % rows), c = (int)(e / rows);
    out[e] = cconj(V[(int64_t)r * ldv + c]);
  }
}
// out[:, j] = U[:, j] * s[j], j < cols
__global__ void scale_cols_kernel(int rows, int cols, const cd* U, const double* s, cd* out) {
  const int64_t total = (int64_t)rows * cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / rows);
    out[e] = cmk(U[e].x * s[c], U[e].y * s[c]);
  }
}

}  // namespace

// Right-to-left truncating SVD sweep of a left-canonical MPS: at site i (dl, d, dr) with the
// carried factor r (dr x b), M = reshape(A_i, dl d, dr) r, svd(reshape(M, dl, d b)) = u s v',
// s <- s[s > 0], dnew = min(#{cumsum(s^2 / sum s^2) < 1 - tol} + 1, dmax), err_trim_i = the
// dropped weight, ent_i = -2 sum s^2 log s, new A_i = reshape(v[:, 1:dnew]', dnew, d, b),
// r = u[:, 1:dnew] diag(s[1:dnew]).  err_glob = 1 - |r|^2 at the end.  The new sites land in
// context scratch at the old sites' offsets (no site grows); dims_out are the new bonds.
int compression_svd(mpsb_ctx* ctx, const mpsb_mps* in, int dmax, double tol, std::vector<int64_t>& dims_out,
                    cd** sites, double* err_glob, double* err_trim, double* ent_ent) {
  if (!ctx || !in || dmax < 1 || !(tol >= 0)) return MPSB_ERR_INVALID_ARG;
  const int na = in->na, d = in->d;
  cudaStream_t st = ctx->stream;
  int64_t maxsite = 1, maxr = 1;
  for (int k = 0; k < na; ++k) {
    maxsite = std::max<int64_t>(maxsite, in->site_elems(k));
    maxr = std::max<int64_t>(maxr, in->dims[k] * in->dims[k]);
  }
  // scratch: new sites (old total), r, M, U, V, dS
  cd* base = nullptr;
  const size_t need = (size_t)in->total + 2 * maxr + 3 * maxsite + maxsite / 2 + 64;
  MPSB_TRY(ensure_slot(ctx, SLOT_MISC, need * sizeof(cd), &base));
  cd* out = base;
  cd* r = out + in->total;
  cd* r2 = r + maxr;
  cd* M = r2 + maxr;
  cd* U = M + maxsite;
  cd* V = U + maxsite;
  double* dS = reinterpret_cast<double*>(V + maxsite);
  dims_out.assign(na + 1, 1);
  MPSB_TRY(set_boundary(ctx, r, cmk(1.0, 0.0)));
  int b = 1;   // current right bond (after truncation)
  std::vector<double> S;
  for (int i = na - 1; i >= 0; --i) {
    const int dl = (int)in->dims[i], dr = (int)in->dims[i + 1];
    {  // M (dl d x b) = A_i (dl d x dr) r (dr x b)
      Gemm g;
      g.M = dl * d; g.N = b; g.K = dr;
      g.A = in->site(i); g.a_m = 1; g.a_k = (int64_t)dl * d;
      g.B = r; g.b_k = 1; g.b_n = dr;
      g.C = M; g.c_m = 1; g.c_n = (int64_t)dl * d;
      MPSB_TRY(run_gemm(ctx, g));
    }
    const int mm = dl, nn = d * b, k = std::min(mm, nn);
    S.assign(k, 0.0);
    MPSB_TRY(svd_launch(mm, nn, M, 1, mm, U, 1, mm, S.data(), V, 1, nn, &ctx->ws, st));
    int kp = 0;
    double stot = 0.0, ent = 0.0;
    while (kp < k && S[kp] > 0) {
      stot += S[kp] * S[kp];
      ent += S[kp] * S[kp] * std::log(S[kp]);
      ++kp;
    }
    if (kp == 0) {
      set_last_message("compressionSVD: site %d is zero", i + 1);
      return MPSB_ERR_NONFINITE;
    }
    int below = 0;
    double cum = 0.0;
    for (int j = 0; j < kp; ++j) {
      cum += S[j] * S[j] / stot;
      if (cum < 1.0 - tol) ++below;
    }
    // below + 1 can exceed the number of positive singular values when tol is below the rounding
    // of the cumulative sum (the reference then fails on v[:, 1:dnew]); keep them all instead
    const int dnew = std::min(std::min(below + 1, dmax), kp);
    double dropped = 0.0;
    for (int j = dnew; j < kp; ++j) dropped += S[j] * S[j];
    if (err_trim) err_trim[i] = dropped / stot;
    if (ent_ent) ent_ent[i] = -2.0 * ent;
    // new site i = v[:, 1:dnew]' as (dnew, d, b); r = u[:, 1:dnew] diag(s)
    count_launch(&ctx->ws);
    adjoint_cols_kernel<<<148 * 2, 256, 0, st>>>(dnew, nn, V, nn, out + in->off[i]);
    MPSB_CUDA_TRY(cudaGetLastError());
    MPSB_CUDA_TRY(cudaMemcpyAsync(dS, S.data(), dnew * sizeof(double), cudaMemcpyHostToDevice, st));
    count_launch(&ctx->ws);
    scale_cols_kernel<<<148 * 2, 256, 0, st>>>(mm, dnew, U, dS, r2);
    MPSB_CUDA_TRY(cudaGetLastError());
    std::swap(r, r2);
    dims_out[i] = dnew;
    b = dnew;
  }
  cd r0;
  MPSB_CUDA_TRY(cudaMemcpyAsync(&r0, r, sizeof(cd), cudaMemcpyDeviceToHost, st));
  MPSB_CUDA_TRY(cudaStreamSynchronize(st));
  if (err_glob) *err_glob = 1.0 - (r0.x * r0.x + r0.y * r0.y);
  *sites = out;
  return MPSB_OK;
}

}  // namespace mpsb

// ---- two-site variational compression with SVD truncation -------------------------------
namespace mpsb {
namespace {

// D[:, j] = s[j] * ... : out (k x n) = diag(s) V^H for the first k columns of V (n x kv)
__global__ void sv_adjoint_kernel(int k, int n, const cd* V, int64_t ldv, const double* s, cd* out) {
  const int64_t total = (int64_t)k * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    const cd v = cconj(V[(int64_t)r * ldv + c]);
    out[e] = s ? cmk(v.x * s[r], v.y * s[r]) : v;
  }
}

int truncation_rule(const std::vector<double>& S, int k, double tol, int dlim) {
  int kp = 0;
  double stot = 0.0;
  while (kp < k && S[kp] > 0) {
    stot += S[kp] * S[kp];
    ++kp;
  }
  if (kp == 0) return 0;
  int below = 0;
  double cum = 0.0;
  for (int j = 0; j < kp; ++j) {
    cum += S[j] * S[j] / stot;
    if (cum < 1.0 - tol) ++below;
  }
  return std::min(std::min(below + 1, dlim), kp);
}

}  // namespace

// compress_sum_var_apply_H_two_site (src/compression.jl:1072-1157) and its relatives: the
// two-site variational compression of  sum_l coef[l] A[l]  (+ coef[numv-1] H A[numv-1] when H
// is given) with guess Ain.  Each pair's effective tensor is
//   av[a0,s1,s2,b0] = sum_l FL_l[a0,a] A_l1[a,s1,c] A_l2[c,s2,b] FR_l[b,b0]
//                   + sum conj(L[a,w,a0]) A1[a,t1,c] O1[w,s1,v,t1] A2[c,t2,b] O2[v,s2,u,t2] R[b,u,b0]
// (the 2-index left environment contracted on its A index and the 3-index one conjugated,
// as every single-site contraction uses them), split by a thin SVD and truncated by the
// compressionSVD! rule (svd_tol, dlim).  mode 0: maxsweeps sweep pairs (R->L then L->R, the
// coefficients on the right boundary); mode 1: one R->L half sweep (the _left form, last site
// U diag(S)); mode 2: one L->R half sweep from right environments of a right-canonical guess
// (the _right form, coefficients on the left boundary, last site diag(S) V').  Bond dims
// change; the result lands in context scratch (site k at offs[k]) with dims_out.  The terms
// may have different bond dims (the stages of a two-site RK4 step do).
int compress_two_site_sum(mpsb_ctx* ctx, const mpsb_mps* Ain, int numv, const cd* coef, const mpsb_mps* const* Av,
                          const mpsb_mpo* H, int maxsweeps, double svd_tol, int dlim, int mode,
                          std::vector<int64_t>& dims_out, std::vector<int64_t>& offs, cd** sites) {
  if (!ctx || !Ain || numv < 1 || !coef || !Av || maxsweeps < 1 || dlim < 1 || !(svd_tol >= 0) || mode < 0 ||
      mode > 2)
    return MPSB_ERR_INVALID_ARG;
  const bool hasH = H != nullptr;
  const int np = hasH ? numv - 1 : numv;   // plain terms
  if (np > 8) return MPSB_ERR_UNSUPPORTED;
  for (int l = 0; l < numv; ++l)
    if (!Av[l]) return MPSB_ERR_INVALID_ARG;
  const mpsb_mps* A = Av[numv - 1];
  const int na = A->na, d = A->d;
  if (Ain->na != na || Ain->d != d || na < 2) return MPSB_ERR_DIMENSION;
  if (hasH && (H->na != na || H->d != d)) return MPSB_ERR_DIMENSION;
  for (int l = 0; l < numv; ++l)
    if (Av[l]->na != na || Av[l]->d != d) return MPSB_ERR_DIMENSION;
  cudaStream_t st = ctx->stream;
  auto bond_over_capacity = [](int b, int v, int64_t c) {   // cannot happen: cap bounds every pair
    set_last_message("two-site compression: bond %d would be %d above its capacity %lld", b, v, (long long)c);
    return MPSB_ERR_UNSUPPORTED;
  };
  std::vector<int64_t> dims = Ain->dims, cap(dims);
  // capacity of bond k: the largest value the sweeps can give it.  A pair's new bond is at most
  // min(bond[k-1] d, d bond[k+1], dlim), so the capacities are the smallest fixed point of
  // cap[k] = max(guess[k], min(dlim, cap[k-1] d, d cap[k+1])) (monotone, bounded by
  // max(guess, dlim)); a guess whose bonds exceed the dims rule raises its neighbours' capacity
  // instead of being cut.
  for (bool changed = true; changed;) {
    changed = false;
    for (int k = 1; k < na; ++k) {
      const int64_t c = std::max<int64_t>(dims[k], std::min<int64_t>(dlim, std::min(cap[k - 1] * d, cap[k + 1] * d)));
      if (c != cap[k]) { cap[k] = c; changed = true; }
    }
  }
  auto DA = [&](int k) { return (int)A->dims[k]; };
  auto DL = [&](int l, int k) { return (int)Av[l]->dims[k]; };   // bond k of plain term l
  auto W = [&](int k) { return hasH ? (int)H->w[k] : 1; };
  // scratch: A0 sites at capacity, the FL / FR stacks (3-index for the H term, 2-index for each
  // plain term), two contraction buffers, the pair tensor and the SVD factors
  offs.assign(na, 0);
  int64_t tot = 0, envtot = 0, env2tot = 0, pairmax = 1, aor = 1;
  std::vector<int64_t> eoff(na + 1), e2off((size_t)np * (na + 1));
  for (int k = 0; k < na; ++k) {
    offs[k] = tot;
    tot += cap[k] * d * cap[k + 1];
  }
  for (int k = 0; k <= na; ++k) {
    eoff[k] = envtot;
    envtot += (int64_t)DA(k) * W(k) * cap[k];
  }
  for (int l = 0; l < np; ++l)   // plain term l: its FL then its FR stack
    for (int k = 0; k <= na; ++k) {
      e2off[(size_t)l * (na + 1) + k] = env2tot;
      env2tot += 2 * (int64_t)DL(l, k) * cap[k];
    }
  for (int l = 0; l < np; ++l) {   // the plain terms' contraction temporaries
    for (int k = 0; k + 1 < na; ++k) {
      aor = std::max<int64_t>(aor, (int64_t)DL(l, k) * d * d * cap[k + 2]);
      aor = std::max<int64_t>(aor, (int64_t)DL(l, k + 1) * d * cap[k + 2]);
    }
    for (int k = 0; k < na; ++k) {
      aor = std::max<int64_t>(aor, (int64_t)DL(l, k) * d * cap[k + 1]);
      aor = std::max<int64_t>(aor, (int64_t)cap[k] * d * DL(l, k + 1));
    }
  }
  for (int k = 0; k + 1 < na; ++k) {
    pairmax = std::max<int64_t>(pairmax, cap[k] * d * d * cap[k + 2]);
    aor = std::max<int64_t>(aor, (int64_t)DA(k) * W(k) * d * d * cap[k + 2]);
    aor = std::max<int64_t>(aor, (int64_t)DA(k + 1) * W(k + 1) * d * cap[k + 2]);
  }
  for (int k = 0; k < na; ++k) {
    aor = std::max<int64_t>(aor, (int64_t)DA(k) * W(k) * d * cap[k + 1]);
    aor = std::max<int64_t>(aor, (int64_t)cap[k] * d * DA(k + 1) * W(k + 1));
  }
  const size_t need = (size_t)tot + 2 * (hasH ? envtot : 0) + (size_t)env2tot + 2 * aor + 3 * pairmax + pairmax / 2 + 64;
  cd* base = nullptr;
  MPSB_TRY(ensure_slot(ctx, SLOT_MISC, need * sizeof(cd), &base));
  cd* A0 = base;
  cd* FLb = A0 + tot;
  cd* FRb = FLb + (hasH ? envtot : 0);
  cd* F2b = FRb + (hasH ? envtot : 0);   // the plain terms' stacks (e2off)
  cd* X = F2b + env2tot;
  cd* Y = X + aor;
  cd* av = Y + aor;
  cd* U = av + pairmax;
  cd* V = U + pairmax;
  double* dS = reinterpret_cast<double*>(V + pairmax);
  auto FL = [&](int k) { return FLb + eoff[k]; };
  auto FR = [&](int k) { return FRb + eoff[k]; };
  auto FL2 = [&](int l, int k) { return F2b + e2off[(size_t)l * (na + 1) + k]; };
  auto FR2 = [&](int l, int k) { return FL2(l, k) + (int64_t)DL(l, k) * cap[k]; };
  auto site0 = [&](int k) { return A0 + offs[k]; };
  const cd ONE_ = cmk(1.0, 0.0), ZERO_ = cmk(0.0, 0.0);
  for (int k = 0; k < na; ++k)   // A0 starts as the guess (dims of Ain)
    MPSB_CUDA_TRY(cudaMemcpyAsync(site0(k), Ain->site(k), Ain->site_elems(k) * sizeof(cd), cudaMemcpyDeviceToDevice, st));

  // environment updates from site k of A0 (bond dims a0 -> a1 of A0)
  auto left_update = [&](int k, int a0, int a1) -> int {   // FL[k+1] from FL[k]
    for (int l = 0; l < np; ++l) {
      MPSB_TRY(op_L2_A3(ctx, FL2(l, k), Av[l]->site(k), X, a0, DL(l, k), d * DL(l, k + 1), ONE_, ZERO_, false));
      MPSB_TRY(op_update_lenv(ctx, site0(k), X, FL2(l, k + 1), a0 * d, a1, DL(l, k + 1), true));
    }
    if (hasH) {
      MPSB_TRY(op_prod_AOL(ctx, A->site(k), H->site(k), FL(k), Y, DA(k), d, DA(k + 1), W(k), W(k + 1), a0));
      MPSB_TRY(op_update_le(ctx, site0(k), Y, FL(k + 1), a0, d, DA(k + 1), W(k + 1), a1));
    }
    return MPSB_OK;
  };
  auto right_update = [&](int k, int a0, int a1) -> int {   // FR[k] from FR[k+1]
    for (int l = 0; l < np; ++l) {
      MPSB_TRY(op_A3_R2(ctx, Av[l]->site(k), FR2(l, k + 1), X, DL(l, k) * d, DL(l, k + 1), a1, ONE_, ZERO_));
      MPSB_TRY(op_update_renv(ctx, site0(k), X, FR2(l, k), DL(l, k), a0, d * a1));
    }
    if (hasH) {
      MPSB_TRY(op_prod_AOR(ctx, A->site(k), H->site(k), FR(k + 1), X, DA(k), d, DA(k + 1), W(k), W(k + 1), a1));
      MPSB_TRY(op_update_re(ctx, site0(k), X, FR(k), DA(k), W(k), d, a1, a0));
    }
    return MPSB_OK;
  };
  // boundaries: the coefficients sit on the right end, or on the left end for mode 2
  for (int l = 0; l < np; ++l) {
    MPSB_TRY(set_boundary(ctx, FL2(l, 0), mode == 2 ? coef[l] : ONE_));
    MPSB_TRY(set_boundary(ctx, FR2(l, na), mode == 2 ? ONE_ : coef[l]));
  }
  if (hasH) {
    // the 3-index left environment is stored conjugated: conj(coef) there applies coef
    MPSB_TRY(set_boundary(ctx, FL(0), mode == 2 ? cconj(coef[numv - 1]) : ONE_));
    MPSB_TRY(set_boundary(ctx, FR(na), mode == 2 ? ONE_ : coef[numv - 1]));
  }
  if (mode == 2) {
    for (int k = na - 1; k >= 2; --k) MPSB_TRY(right_update(k, (int)dims[k], (int)dims[k + 1]));
  } else {
    for (int k = 0; k < na - 2; ++k) MPSB_TRY(left_update(k, (int)dims[k], (int)dims[k + 1]));
  }
  std::vector<double> S;
  // the pair tensor of sites (j, j+1) into av: (dims[j] d) x (d dims[j+2])
  auto pair = [&](int j) -> int {
    const int b0 = (int)dims[j + 2], a0 = (int)dims[j];
    for (int l = 0; l < np; ++l) {
      // X[c, s2, b0] = A_l[j+1] FR_l[j+2];  Y[a, s1, (s2 b0)] = A_l[j] X;  av (+)= FL_l[j] Y
      MPSB_TRY(op_A3_R2(ctx, Av[l]->site(j + 1), FR2(l, j + 2), X, DL(l, j + 1) * d, DL(l, j + 2), b0, ONE_, ZERO_));
      MPSB_TRY(op_A3_R2(ctx, Av[l]->site(j), X, Y, DL(l, j) * d, DL(l, j + 1), d * b0, ONE_, ZERO_));
      MPSB_TRY(op_L2_A3(ctx, FL2(l, j), Y, av, a0, DL(l, j), d * d * b0, ONE_, l ? ONE_ : ZERO_, false));
    }
    if (!hasH) return MPSB_OK;
    // X[c, v, s2, b0] = prod_AOR(A[j+1], H[j+1], FR[j+2])
    MPSB_TRY(op_prod_AOR(ctx, A->site(j + 1), H->site(j + 1), FR(j + 2), X, DA(j + 1), d, DA(j + 2), W(j + 1), W(j + 2), b0));
    // Y[a, w, s1, (s2 b0)] = prod_AOR(A[j], H[j], X as R[c, v, (s2 b0)])
    MPSB_TRY(op_prod_AOR(ctx, A->site(j), H->site(j), X, Y, DA(j), d, DA(j + 1), W(j), W(j + 1), d * b0));
    // av[a0, s1, (s2 b0)] (+)= sum_{a, w} conj(L[a, w, a0]) Y[a, w, s1, (s2 b0)]
    return op_prod_LR_3_4(ctx, FL(j), Y, av, DA(j), W(j), a0, d, d * b0, ONE_, np ? ONE_ : ZERO_);
  };
  auto svd_pair = [&](int j, int& k) -> int {
    const int m = (int)dims[j] * d, n = d * (int)dims[j + 2];
    k = std::min(m, n);
    S.assign(k, 0.0);
    return svd_launch(m, n, av, 1, m, U, 1, m, S.data(), V, 1, n, &ctx->ws, st);
  };
  int k = 0, dnew = 1;
  auto sweep_left = [&]() -> int {   // pairs (j, j+1) from the right end, site j+1 becomes V'
    for (int j = na - 2; j >= 0; --j) {
      MPSB_TRY(pair(j));
      MPSB_TRY(svd_pair(j, k));
      dnew = truncation_rule(S, k, svd_tol, dlim);
      if (dnew > cap[j + 1]) return bond_over_capacity(j + 1, dnew, cap[j + 1]);
      if (dnew == 0) { set_last_message("two-site compression: zero pair tensor"); return MPSB_ERR_NONFINITE; }
      dims[j + 1] = dnew;
      const int n = d * (int)dims[j + 2];
      count_launch(&ctx->ws);
      sv_adjoint_kernel<<<148 * 2, 256, 0, st>>>(dnew, n, V, n, nullptr, site0(j + 1));
      MPSB_CUDA_TRY(cudaGetLastError());
      MPSB_TRY(right_update(j + 1, dnew, (int)dims[j + 2]));
    }
    return MPSB_OK;
  };
  auto sweep_right = [&]() -> int {   // pairs from the left end, site j becomes U
    for (int j = 0; j <= na - 2; ++j) {
      MPSB_TRY(pair(j));
      MPSB_TRY(svd_pair(j, k));
      dnew = truncation_rule(S, k, svd_tol, dlim);
      if (dnew > cap[j + 1]) return bond_over_capacity(j + 1, dnew, cap[j + 1]);
      if (dnew == 0) { set_last_message("two-site compression: zero pair tensor"); return MPSB_ERR_NONFINITE; }
      dims[j + 1] = dnew;
      const int m = (int)dims[j] * d;
      MPSB_CUDA_TRY(cudaMemcpyAsync(site0(j), U, (size_t)m * dnew * sizeof(cd), cudaMemcpyDeviceToDevice, st));
      MPSB_TRY(left_update(j, (int)dims[j], dnew));
    }
    return MPSB_OK;
  };
  // last site of a L->R sweep: diag(S) V' of the last pair
  auto close_right = [&]() -> int {
    const int n = d * (int)dims[na];
    MPSB_CUDA_TRY(cudaMemcpyAsync(dS, S.data(), dnew * sizeof(double), cudaMemcpyHostToDevice, st));
    count_launch(&ctx->ws);
    sv_adjoint_kernel<<<148 * 2, 256, 0, st>>>(dnew, n, V, n, dS, site0(na - 1));
    MPSB_CUDA_TRY(cudaGetLastError());
    return MPSB_OK;
  };
  if (mode == 0) {
    for (int sweep = 0; sweep < maxsweeps; ++sweep) {
      MPSB_TRY(sweep_left());
      MPSB_TRY(sweep_right());
      MPSB_TRY(close_right());
    }
  } else if (mode == 1) {
    MPSB_TRY(sweep_left());
    // first site: U diag(S) of the last pair
    const int m = (int)dims[0] * d;
    MPSB_CUDA_TRY(cudaMemcpyAsync(dS, S.data(), dnew * sizeof(double), cudaMemcpyHostToDevice, st));
    count_launch(&ctx->ws);
    scale_cols_kernel<<<148 * 2, 256, 0, st>>>(m, dnew, U, dS, site0(0));
    MPSB_CUDA_TRY(cudaGetLastError());
  } else {
    MPSB_TRY(sweep_right());
    MPSB_TRY(close_right());
  }
  dims_out = dims;
  *sites = A0;
  return MPSB_OK;
}

// compress_var_apply_H_two_site (src/compression.jl:355-411): one term through H, coefficient 1
int compress_two_site(mpsb_ctx* ctx, const mpsb_mps* Ain, const mpsb_mps* A, const mpsb_mpo* H, int maxsweeps,
                      double svd_tol, int dlim, std::vector<int64_t>& dims_out, std::vector<int64_t>& offs,
                      cd** sites) {
  if (!H) return MPSB_ERR_INVALID_ARG;
  const cd one = cmk(1.0, 0.0);
  const mpsb_mps* terms[1] = {A};
  return compress_two_site_sum(ctx, Ain, 1, &one, terms, H, maxsweeps, svd_tol, dlim, 0, dims_out, offs, sites);
}

}  // namespace mpsb
