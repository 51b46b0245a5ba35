// ground_state_search! (src/groundstate.jl:67-147): single-site variational sweeps, each site
// solved for the lowest eigenpair of the effective operator applied as A_prod_LOR_eigs
// (src/MatrixProductStates.jl:246-253): out[a0,s,b0] = sum L[a,w,a0] A[a,s',b] O[w,s,w',s'] R[b,w',b0],
// with the left environments as update_le stores them (conjugated) and used unconjugated.
//
// The reference calls ARPACK `eigs(nev=1, which=:SR, v0=site, tol)`, which is absent here; the
// eigensolver is Lanczos with full (twice-applied classical Gram-Schmidt) reorthogonalisation
// on device vectors, restarted from the Ritz vector every LZ_KMAX steps, the tridiagonal's
// lowest eigenvalue by Sturm-sequence bisection and its eigenvector by inverse iteration
// (host, O(k)).  Convergence: |beta_k s_k| <= tol max(|theta|, tiny), ARPACK's criterion.
// The eigenvector's phase, arbitrary in ARPACK, is fixed so that <v0|x> is real positive
// (v0 = the site's current tensor), which keeps consecutive sweeps continuous.
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace mpsb {
namespace {

constexpr int LZ_KMAX = 64;
const cd ONE = {1.0, 0.0};
const cd ZERO = {0.0, 0.0};
const cd MONE = {-1.0, 0.0};

__global__ void conj_kernel(cd* x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i].y = -x[i].y;
}
// y = a * x (y may alias x)
__global__ void cscale_kernel(cd* y, const cd* x, int64_t n, cd a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = cmul(a, x[i]);
}

int conj_launch(mpsb_ctx* ctx, cd* x, int64_t n) {
  count_launch(&ctx->ws);
  conj_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 4), 256, 0, ctx->stream>>>(x, n);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}
int scale_launch(mpsb_ctx* ctx, cd* y, const cd* x, int64_t n, cd a) {
  count_launch(&ctx->ws);
  cscale_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 4), 256, 0, ctx->stream>>>(y, x, n, a);
  MPSB_CUDA_TRY(cudaGetLastError());
  return MPSB_OK;
}

// out = V[:, 0:k]^H w  (k values, device) then copied to the host
int project(mpsb_ctx* ctx, const cd* V, int64_t n, int k, const cd* w, cd* dh, std::vector<cd>& h) {
  Gemm g;
  g.M = k; g.N = 1; g.K = (int)n;
  g.A = V; g.a_m = n; g.a_k = 1; g.conjA = true;
  g.B = w; g.b_k = 1; g.b_n = n;
  g.C = dh; g.c_m = 1; g.c_n = k;
  MPSB_TRY(run_gemm(ctx, g));
  h.resize(k);
  MPSB_CUDA_TRY(cudaMemcpyAsync(h.data(), dh, k * sizeof(cd), cudaMemcpyDeviceToHost, ctx->stream));
  MPSB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MPSB_OK;
}

// w += alpha * V[:, 0:k] c  (c on the device)
int combine(mpsb_ctx* ctx, const cd* V, int64_t n, int k, const cd* dc, cd* w, cd alpha, cd beta) {
  Gemm g;
  g.M = (int)n; g.N = 1; g.K = k;
  g.A = V; g.a_m = 1; g.a_k = n;
  g.B = dc; g.b_k = 1; g.b_n = k;
  g.C = w; g.c_m = 1; g.c_n = n;
  g.alpha = alpha; g.beta = beta;
  return run_gemm(ctx, g);
}

// Lowest eigenpair of the symmetric tridiagonal (a[0..k), b[0..k-1)): bisection on the Sturm
// count, then inverse iteration (Thomas algorithm) for the eigenvector (unit 2-norm).
double tridiag_lowest(const std::vector<double>& a, const std::vector<double>& b, int k, std::vector<double>& s) {
  double lo = a[0], hi = a[0];
  for (int i = 0; i < k; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < k ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto count_below = [&](double x) {
    int c = 0;
    double q = a[0] - x;
    if (q < 0) ++c;
    for (int i = 1; i < k; ++i) {
      const double qq = (q == 0.0) ? 1e-300 : q;
      q = a[i] - x - b[i - 1] * b[i - 1] / qq;
      if (q < 0) ++c;
    }
    return c;
  };
  for (int it = 0; it < 200 && hi - lo > 2e-16 * std::max(std::fabs(lo), std::fabs(hi)) + 1e-300; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= 1) hi = mid;
    else lo = mid;
  }
  const double theta = 0.5 * (lo + hi);
  // inverse iteration with (T - theta') y = s, theta' just below theta
  const double shift = theta - 1e-14 * std::max(1.0, std::fabs(theta));
  s.assign(k, 1.0);
  std::vector<double> c(k), d(k);
  for (int pass = 0; pass < 3; ++pass) {
    // forward elimination on the tridiagonal (diag a - shift, off b)
    double den = a[0] - shift;
    if (den == 0.0) den = 1e-300;
    c[0] = (k > 1 ? b[0] : 0.0) / den;
    d[0] = s[0] / den;
    for (int i = 1; i < k; ++i) {
      den = a[i] - shift - b[i - 1] * c[i - 1];
      if (den == 0.0) den = 1e-300;
      c[i] = (i + 1 < k ? b[i] : 0.0) / den;
      d[i] = (s[i] - b[i - 1] * d[i - 1]) / den;
    }
    s[k - 1] = d[k - 1];
    for (int i = k - 2; i >= 0; --i) s[i] = d[i] - c[i] * s[i + 1];
    double nrm = 0.0;
    for (int i = 0; i < k; ++i) nrm += s[i] * s[i];
    nrm = std::sqrt(nrm);
    for (int i = 0; i < k; ++i) s[i] /= nrm;
  }
  return theta;
}

struct SiteOp {   // the effective operator of one site: FL (bond j), H[j], FR (bond j+1)
  const cd* FL; const cd* O; const cd* FR;
  int Dl, d, Dr, wl, wr;
  cd* AOR;
};

int apply_site(mpsb_ctx* ctx, const SiteOp& so, const cd* x, cd* out) {
  MPSB_TRY(op_prod_AOR(ctx, x, so.O, so.FR, so.AOR, so.Dl, so.d, so.Dr, so.wl, so.wr, so.Dr));
  Gemm g;   // out[a0, (s, b0)] = sum_{(a, w)} L[(a, w), a0] AOR[(a, w), (s, b0)]  (L not conjugated)
  g.M = so.Dl; g.N = so.d * so.Dr; g.K = so.Dl * so.wl;
  g.A = so.FL; g.a_m = (int64_t)so.Dl * so.wl; g.a_k = 1;
  g.B = so.AOR; g.b_k = 1; g.b_n = (int64_t)so.Dl * so.wl;
  g.C = out; g.c_m = 1; g.c_n = so.Dl;
  return run_gemm(ctx, g);
}

// x (device, n): start vector in, lowest eigenvector out.  V holds LZ_KMAX + 1 basis vectors,
// w one more, dh LZ_KMAX + 1 coefficients.
int lanczos_lowest(mpsb_ctx* ctx, const SiteOp& so, int64_t n, cd* x, cd* V, cd* w, cd* dh, double tol, int maxiter,
                   double* theta_out) {
  std::vector<cd> h, h2;
  std::vector<double> al, be, sv;
  int iters = 0;
  double theta = 0.0;
  for (;;) {
    MPSB_TRY(project(ctx, x, n, 1, x, dh, h));
    double nrm = std::sqrt(std::max(0.0, h[0].x));
    if (nrm == 0.0) {   // a zero start vector: start from the first unit vector
      MPSB_CUDA_TRY(cudaMemsetAsync(x, 0, n * sizeof(cd), ctx->stream));
      MPSB_TRY(set_boundary(ctx, x, ONE));
      nrm = 1.0;
    }
    MPSB_TRY(scale_launch(ctx, V, x, n, cmk(1.0 / nrm, 0.0)));
    al.clear();
    be.clear();
    int k = 0;
    bool done = false;
    for (;;) {
      cd* vk = V + (int64_t)k * n;
      MPSB_TRY(apply_site(ctx, so, vk, w));
      ++iters;
      // two passes of classical Gram-Schmidt against V[:, 0..k]
      MPSB_TRY(project(ctx, V, n, k + 1, w, dh, h));
      MPSB_TRY(combine(ctx, V, n, k + 1, dh, w, MONE, ONE));
      MPSB_TRY(project(ctx, V, n, k + 1, w, dh, h2));
      MPSB_TRY(combine(ctx, V, n, k + 1, dh, w, MONE, ONE));
      al.push_back(h[k].x + h2[k].x);
      std::vector<cd> nn;
      MPSB_TRY(project(ctx, w, n, 1, w, dh, nn));
      const double beta = std::sqrt(std::max(0.0, nn[0].x));
      theta = tridiag_lowest(al, be, k + 1, sv);
      const double res = std::fabs(beta * sv[k]);
      const bool conv = res <= tol * std::max(std::fabs(theta), 1e-300) || beta <= 1e-14 * (std::fabs(theta) + 1e-300);
      if (conv || k + 1 >= n) done = true;
      if (done || iters >= maxiter || k + 1 >= LZ_KMAX) break;
      be.push_back(beta);
      MPSB_TRY(scale_launch(ctx, V + (int64_t)(k + 1) * n, w, n, cmk(1.0 / beta, 0.0)));
      ++k;
    }
    // Ritz vector x = V s, phase fixed by <v0|x> = s[0] > 0 (sign of the real s)
    std::vector<cd> sc(k + 1);
    const double sg = sv[0] < 0 ? -1.0 : 1.0;
    for (int i = 0; i <= k; ++i) sc[i] = cmk(sg * sv[i], 0.0);
    MPSB_CUDA_TRY(cudaMemcpyAsync(dh, sc.data(), (k + 1) * sizeof(cd), cudaMemcpyHostToDevice, ctx->stream));
    MPSB_TRY(combine(ctx, V, n, k + 1, dh, x, ONE, ZERO));
    if (done || iters >= maxiter) break;
  }
  *theta_out = theta;
  return MPSB_OK;
}

}  // namespace

int ground_state_search(mpsb_ctx* ctx, mpsb_mps* At, const mpsb_mpo* H, int maxsweeps, double converge_rat,
                        double eigs_tol, double* ae_out) {
  if (!ctx || !At || !H || maxsweeps < 0 || !(eigs_tol >= 0)) return MPSB_ERR_INVALID_ARG;
  const int na = At->na, d = At->d;
  if (H->na != na || H->d != d) return MPSB_ERR_DIMENSION;
  auto D = [&](int k) { return (int)At->dims[k]; };
  auto W = [&](int k) { return (int)H->w[k]; };
  // environments FL and FR at every bond, the site-op intermediates, the Lanczos basis
  std::vector<int64_t> eoff(na + 1);
  int64_t etot = 0, nmax = 1, aor = 1, rv = 1;
  for (int k = 0; k <= na; ++k) {
    eoff[k] = etot;
    etot += (int64_t)D(k) * W(k) * D(k);
  }
  for (int k = 0; k < na; ++k) {
    nmax = std::max<int64_t>(nmax, (int64_t)D(k) * d * D(k + 1));
    aor = std::max<int64_t>(aor, (int64_t)D(k) * W(k) * d * D(k + 1));
    aor = std::max<int64_t>(aor, (int64_t)D(k) * d * D(k + 1) * W(k + 1));
    rv = std::max<int64_t>(rv, (int64_t)D(k) * D(k));
  }
  cd* env = nullptr;
  MPSB_TRY(ensure_slot(ctx, SLOT_GSENV, 2 * etot * sizeof(cd), &env));
  cd* FLb = env;
  cd* FRb = env + etot;
  auto FL = [&](int k) { return FLb + eoff[k]; };
  auto FR = [&](int k) { return FRb + eoff[k]; };
  const size_t nvec = (size_t)nmax * (LZ_KMAX + 2) + aor + rv + nmax + (LZ_KMAX + 2);
  cd* vec = nullptr;
  MPSB_TRY(ensure_slot(ctx, SLOT_GSVEC, nvec * sizeof(cd), &vec));
  cd* V = vec;
  cd* w = V + (int64_t)nmax * (LZ_KMAX + 1);
  cd* AOR = w + nmax;
  cd* R = AOR + aor;
  cd* tmp = R + rv;
  cd* dh = tmp + nmax;
  cd* AOL = nullptr;
  MPSB_TRY(ensure_slot(ctx, SLOT_AOL, aor * sizeof(cd), &AOL));

  auto site_op = [&](int j) {
    SiteOp so;
    so.FL = FL(j); so.O = H->site(j); so.FR = FR(j + 1);
    so.Dl = D(j); so.d = d; so.Dr = D(j + 1); so.wl = W(j); so.wr = W(j + 1);
    so.AOR = AOR;
    return so;
  };
  auto update_fl = [&](int j) -> int {   // FL[j+1] = update_le(At[j], H[j], At[j], FL[j])
    MPSB_TRY(op_prod_AOL(ctx, At->site(j), H->site(j), FL(j), AOL, D(j), d, D(j + 1), W(j), W(j + 1), D(j)));
    return op_update_le(ctx, At->site(j), AOL, FL(j + 1), D(j), d, D(j + 1), W(j + 1), D(j + 1));
  };
  auto update_fr = [&](int j) -> int {   // FR[j] = update_re(At[j], H[j], At[j], FR[j+1])
    MPSB_TRY(op_prod_AOR(ctx, At->site(j), H->site(j), FR(j + 1), AOR, D(j), d, D(j + 1), W(j), W(j + 1), D(j + 1)));
    return op_update_re(ctx, At->site(j), AOR, FR(j), D(j), W(j), d, D(j + 1), D(j));
  };
  const int maxiter = 1000;
  auto solve = [&](int j, double* ae) -> int {
    return lanczos_lowest(ctx, site_op(j), (int64_t)D(j) * d * D(j + 1), At->site(j), V, w, dh, eigs_tol, maxiter, ae);
  };

  MPSB_TRY(set_boundary(ctx, FL(0), ONE));
  for (int j = 0; j < na - 1; ++j) MPSB_TRY(update_fl(j));
  MPSB_TRY(set_boundary(ctx, FR(na), ONE));
  double ae = 0.0, aestart = 0.0;
  for (int sweep = 0; sweep < maxsweeps; ++sweep) {
    for (int j = na - 1; j >= 1; --j) {   // sweep left
      MPSB_TRY(solve(j, &ae));
      if (j == na - 1) aestart = ae;
      // QR of the adjoint of reshape(av, Dl, d Dr): At[j] = Q', R absorbed as At[j-1] R.'
      const int Dl = D(j), Dr = D(j + 1);
      cd* a = At->site(j);
      MPSB_TRY(conj_launch(ctx, a, (int64_t)Dl * d * Dr));
      QrProblem p;
      p.m = d * Dr; p.n = Dl;
      p.X = a; p.x_r = Dl; p.x_c = 1;
      p.Q = a; p.q_r = Dl; p.q_c = 1;
      p.R = R; p.r_r = 1; p.r_c = Dl;
      p.err = ctx->err();
      MPSB_TRY(run_qr(ctx, p));
      MPSB_TRY(conj_launch(ctx, a, (int64_t)Dl * d * Dr));
      MPSB_TRY(update_fr(j));
      {  // At[j-1][x, c] = sum_b At[j-1][x, b] R[c, b]
        const int M = D(j - 1) * d;
        Gemm g;
        g.M = M; g.N = Dl; g.K = Dl;
        g.A = At->site(j - 1); g.a_m = 1; g.a_k = M;
        g.B = R; g.b_k = Dl; g.b_n = 1;
        g.C = tmp; g.c_m = 1; g.c_n = M;
        MPSB_TRY(run_gemm(ctx, g));
        count_launch(&ctx->ws);
        MPSB_TRY(copy(At->site(j - 1), tmp, (int64_t)M * Dl, ctx->stream));
      }
    }
    for (int j = 0; j < na - 1; ++j) {   // sweep right
      MPSB_TRY(solve(j, &ae));
      const int Dl = D(j), Dr = D(j + 1);
      MPSB_TRY(op_orth_left(ctx, At->site(j), Dl, d, Dr, R));
      MPSB_TRY(update_fl(j));
      {  // At[j+1][c, s, e] = sum_b R[c, b] At[j+1][b, s, e]
        const int N = d * D(j + 2);
        Gemm g;
        g.M = Dr; g.N = N; g.K = Dr;
        g.A = R; g.a_m = 1; g.a_k = Dr;
        g.B = At->site(j + 1); g.b_k = 1; g.b_n = Dr;
        g.C = tmp; g.c_m = 1; g.c_n = Dr;
        MPSB_TRY(run_gemm(ctx, g));
        count_launch(&ctx->ws);
        MPSB_TRY(copy(At->site(j + 1), tmp, (int64_t)Dr * N, ctx->stream));
      }
    }
    MPSB_TRY(solve(na - 1, &ae));
    if (std::fabs(ae) > converge_rat * std::fabs(aestart) || std::fabs(ae) < 1e-10) break;
  }
  if (ae_out) *ae_out = ae;
  return MPSB_OK;
}

}  // namespace mpsb
