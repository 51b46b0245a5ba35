// Sweep orchestration: the reference's contraction helpers (src/mps_base.jl), gauge moves
// (src/orthonormalisation.jl) and compression sweeps (src/compression.jl) expressed as
// launches of the strided GEMM, MPO-apply and cluster-QR kernels on the context stream.
#include <algorithm>
#include <cstring>
#include <functional>

#include "engine.cuh"
#include "ozaki.cuh"

namespace mpsb {

// While alive, the sweep contractions of this context run at its configured precision
// (mpsb_ctx_set_precision); outside (observables, gauge moves, eigen-solvers) they are FP64.
struct SplitScope {
  mpsb_ctx* c;
  bool prev;
  explicit SplitScope(mpsb_ctx* ctx) : c(ctx), prev(ctx->split_on) { c->split_on = c->split_slices > 0; }
  ~SplitScope() { c->split_on = prev; }
};

// A scratch slot of `bytes` per copy: in a batched call it holds ctx->batch copies, registered
// with the copy stride cap / batch so that every kernel finds copy b of any pointer into it.
int ensure_slot(mpsb_ctx* ctx, Slot s, size_t bytes, cd** out) {
  DevBuf& b = ctx->ws.named[s];
  void* before = b.p;
  const size_t B = (size_t)std::max(1, ctx->batch);
  MPSB_TRY(devbuf_ensure(&ctx->ws, b, bytes * B));
  if (b.p != before) {
    ctx->ws_generation++;
    if (before) ctx->slabs.erase(reinterpret_cast<uintptr_t>(before));
  }
  const uintptr_t base = reinterpret_cast<uintptr_t>(b.p);
  if (B > 1) ctx->slabs[base] = {base + b.cap, (int64_t)(b.cap / sizeof(cd) / B)};
  else ctx->slabs.erase(base);
  *out = static_cast<cd*>(b.p);
  return MPSB_OK;
}

// The copies of a batched call: every MPS and environment handle of the call must hold the same
// number of copies; a handle created as part of a batch (or a view of one copy) puts the call in
// batched mode (split-K and the sliced-path choice decided per problem), so that a copy computes
// the same bits in a batch of any size.  While alive, kernels of the context run ctx->batch copies.
struct BatchScope {
  mpsb_ctx* c;
  int prev;
  bool prev_ns, prev_ns_side, prev_split;
  BatchScope(mpsb_ctx* ctx, int B, bool batched)
      : c(ctx), prev(ctx->batch), prev_ns(ctx->ws.per_problem), prev_ns_side(ctx->ws_side.per_problem),
        prev_split(ctx->split_on) {
    c->batch = B;
    c->ws.per_problem = c->ws_side.per_problem = batched;
  }
  ~BatchScope() {
    c->batch = prev;
    c->ws.per_problem = prev_ns;
    c->ws_side.per_problem = prev_ns_side;
    c->split_on = prev_split;
  }
};

static int call_batch(std::initializer_list<const mpsb_mps*> mps, std::initializer_list<const mpsb_env*> envs,
                      int* B, bool* batched) {
  *B = -1;
  *batched = false;
  for (const mpsb_mps* m : mps) {
    if (!m) continue;
    if (*B < 0) *B = m->batch;
    if (m->batch != *B) return MPSB_ERR_DIMENSION;
    *batched = *batched || m->batched;
  }
  for (const mpsb_env* e : envs) {
    if (!e) continue;
    if (*B < 0) *B = e->batch;
    if (e->batch != *B) return MPSB_ERR_DIMENSION;
    *batched = *batched || e->batched;
  }
  if (*B < 0) *B = 1;
  return MPSB_OK;
}

// Whether a sweep GEMM takes the sliced path: by its output tiles (a plain call), or -- in a
// batched call, where the decision must not depend on the batch size -- by its own work alone.
static bool split_worth(const mpsb_ctx* ctx, const Gemm& g) {
  if (ctx->ws.per_problem) return 8.0 * g.M * g.N * g.K >= ctx->split_min_flops && g.K >= 16;
  const int64_t tiles = ((int64_t)(g.M + 127) / 128) * ((2 * (int64_t)g.N + 63) / 64);
  return tiles >= ctx->split_min_tiles && g.K >= 16;
}

int run_gemm(mpsb_ctx* ctx, const Gemm& g0) {
  Gemm g = g0;
  if (ctx->batch > 1 && g.batch == 1) {
    g.batch = ctx->batch;
    g.a_b = ctx->stride_of(g.A);
    g.b_b = ctx->stride_of(g.B);
    g.c_b = ctx->stride_of(g.C);
  }
  if (ctx->split_on && ozgemm_supported(g, ctx->split_slices) && split_worth(ctx, g)) {
    void* before_oz = ctx->ws.oz.p;
    MPSB_TRY(devbuf_ensure(&ctx->ws, ctx->ws.oz, ozgemm_scratch_bytes(g, ctx->split_slices)));
    if (ctx->ws.oz.p != before_oz) ctx->ws_generation++;
    return ozgemm_launch(g, ctx->split_slices, ctx->ws.oz.p, ctx->ws.oz.cap, ctx->err(), &ctx->ws, ctx->stream);
  }
  void* before = ctx->ws.splitk.p;
  int st = gemm_launch(g, &ctx->ws, ctx->stream);
  if (ctx->ws.splitk.p != before) ctx->ws_generation++;
  return st;
}

static inline int run_mpo(mpsb_ctx* ctx, const MpoApply& a0, int64_t k1, int64_t k2, int64_t m1, int64_t m2) {
  MpoApply a = a0;
  if (ctx->batch > 1) {
    a.batch = ctx->batch;
    a.in_b = ctx->stride_of(a.in);
    a.op_b = ctx->stride_of(a.op);
    a.out_b = ctx->stride_of(a.out);
  }
  count_launch(&ctx->ws);
  return mpo_apply_launch_strided(a, k1, k2, m1, m2, ctx->stream);
}

static const cd ONE = {1.0, 0.0};
static const cd ZERO = {0.0, 0.0};

// prod_AOR (src/mps_base.jl:7-19): T = A*R (GEMM), AOR = O . T (small-K apply, permutes folded)
int op_prod_AOR(mpsb_ctx* ctx, const cd* A, const cd* O, const cd* R, cd* AOR, int chiL, int d, int chiR, int wL,
                int wR, int chiR0) {
  cd* T;
  MPSB_TRY(ensure_slot(ctx, SLOT_T, (size_t)chiL * d * wR * chiR0 * sizeof(cd), &T));
  Gemm g;
  g.M = chiL * d; g.N = wR * chiR0; g.K = chiR;
  g.A = A; g.a_m = 1; g.a_k = (int64_t)chiL * d;
  g.B = R; g.b_k = 1; g.b_n = chiR;
  g.C = T; g.c_m = 1; g.c_n = (int64_t)chiL * d;
  MPSB_TRY(run_gemm(ctx, g));
  MpoApply a;
  a.X = chiL; a.Y = chiR0; a.K1 = d; a.K2 = wR; a.M1 = wL; a.M2 = d;
  a.in = T; a.in_x = 1; a.in_k1 = chiL; a.in_k2 = (int64_t)chiL * d; a.in_y = (int64_t)chiL * d * wR;
  a.op = O;
  a.out = AOR; a.out_x = 1; a.out_m1 = chiL; a.out_m2 = (int64_t)chiL * wL; a.out_y = (int64_t)chiL * wL * d;
  return run_mpo(ctx, a, (int64_t)wL * d * wR, (int64_t)wL * d, 1, wL);
}

// prod_AOL (src/mps_base.jl:26-39): G1 = L' * A (GEMM), AOL = G1 . O
int op_prod_AOL(mpsb_ctx* ctx, const cd* A, const cd* O, const cd* L, cd* AOL, int chiL, int d, int chiR, int wL,
                int wR, int chiL0) {
  cd* G1;
  MPSB_TRY(ensure_slot(ctx, SLOT_G1, (size_t)wL * chiL0 * d * chiR * sizeof(cd), &G1));
  Gemm g;
  g.M = wL * chiL0; g.N = d * chiR; g.K = chiL;
  g.A = L; g.a_m = chiL; g.a_k = 1; g.conjA = true;
  g.B = A; g.b_k = 1; g.b_n = chiL;
  g.C = G1; g.c_m = 1; g.c_n = (int64_t)wL * chiL0;
  MPSB_TRY(run_gemm(ctx, g));
  MpoApply a;
  a.X = chiL0; a.Y = chiR; a.K1 = wL; a.K2 = d; a.M1 = d; a.M2 = wR;
  a.in = G1; a.in_x = wL; a.in_k1 = 1; a.in_k2 = (int64_t)wL * chiL0; a.in_y = (int64_t)wL * chiL0 * d;
  a.op = O;
  a.out = AOL; a.out_x = 1; a.out_m1 = chiL0; a.out_m2 = (int64_t)chiL0 * d * chiR; a.out_y = (int64_t)chiL0 * d;
  return run_mpo(ctx, a, 1, (int64_t)wL * d * wR, wL, (int64_t)wL * d);
}

// prod_LR!(A0, L, AOR) (src/mps_base.jl:53-61): A0 = L' * AOR
int op_prod_LR_3_4(mpsb_ctx* ctx, const cd* L, const cd* AOR, cd* A0, int chiL, int wL, int chiL0, int d, int chiR0,
                   cd alpha, cd beta) {
  Gemm g;
  g.M = chiL0; g.N = d * chiR0; g.K = chiL * wL;
  g.A = L; g.a_m = (int64_t)chiL * wL; g.a_k = 1; g.conjA = true;
  g.B = AOR; g.b_k = 1; g.b_n = (int64_t)chiL * wL;
  g.C = A0; g.c_m = 1; g.c_n = chiL0;
  g.alpha = alpha; g.beta = beta;
  return run_gemm(ctx, g);
}

// prod_LR!(A0, AOL, R) (src/mps_base.jl:73-81): A0 = AOL * R
int op_prod_LR_4_3(mpsb_ctx* ctx, const cd* AOL, const cd* R, cd* A0, int chiL0, int d, int chiR, int wR, int chiR0,
                   cd alpha, cd beta) {
  Gemm g;
  g.M = chiL0 * d; g.N = chiR0; g.K = chiR * wR;
  g.A = AOL; g.a_m = 1; g.a_k = (int64_t)chiL0 * d;
  g.B = R; g.b_k = 1; g.b_n = (int64_t)chiR * wR;
  g.C = A0; g.c_m = 1; g.c_n = (int64_t)chiL0 * d;
  g.alpha = alpha; g.beta = beta;
  return run_gemm(ctx, g);
}

// update_re!(env, A0, AOR) (src/mps_base.jl:151-160): env = AOR * A0'
int op_update_re(mpsb_ctx* ctx, const cd* A0, const cd* AOR, cd* env, int chiL, int wL, int d, int chiR0, int chiL0) {
  Gemm g;
  g.M = chiL * wL; g.N = chiL0; g.K = d * chiR0;
  g.A = AOR; g.a_m = 1; g.a_k = (int64_t)chiL * wL;
  g.B = A0; g.b_k = chiL0; g.b_n = 1; g.conjB = true;
  g.C = env; g.c_m = 1; g.c_n = (int64_t)chiL * wL;
  return run_gemm(ctx, g);
}

// update_le!(env, A0, AOL) (src/mps_base.jl:232-241): env = AOL' * A0
int op_update_le(mpsb_ctx* ctx, const cd* A0, const cd* AOL, cd* env, int chiL0, int d, int chiR, int wR, int chiR0) {
  Gemm g;
  g.M = chiR * wR; g.N = chiR0; g.K = chiL0 * d;
  g.A = AOL; g.a_m = (int64_t)chiL0 * d; g.a_k = 1; g.conjA = true;
  g.B = A0; g.b_k = 1; g.b_n = (int64_t)chiL0 * d;
  g.C = env; g.c_m = 1; g.c_n = (int64_t)chiR * wR;
  return run_gemm(ctx, g);
}

// prod_LR(L2, A3) (src/mps_base.jl:85-90, 100-108): out(x, rest) = L(x, chiL) * A(chiL, rest);
// transL gives prod_LR_co (L.')
int op_L2_A3(mpsb_ctx* ctx, const cd* L, const cd* A, cd* out, int x, int chiL, int rest, cd alpha, cd beta,
             bool transL) {
  Gemm g;
  g.M = x; g.N = rest; g.K = chiL;
  g.A = L;
  if (transL) { g.a_m = chiL; g.a_k = 1; } else { g.a_m = 1; g.a_k = x; }
  g.B = A; g.b_k = 1; g.b_n = chiL;
  g.C = out; g.c_m = 1; g.c_n = x;
  g.alpha = alpha; g.beta = beta;
  return run_gemm(ctx, g);
}

// prod_LR(A3, R2) (src/mps_base.jl:122-137): out(lead, y) = A(lead, chiR) * R(chiR, y)
int op_A3_R2(mpsb_ctx* ctx, const cd* A, const cd* R, cd* out, int lead, int chiR, int y, cd alpha, cd beta) {
  Gemm g;
  g.M = lead; g.N = y; g.K = chiR;
  g.A = A; g.a_m = 1; g.a_k = lead;
  g.B = R; g.b_k = 1; g.b_n = chiR;
  g.C = out; g.c_m = 1; g.c_n = lead;
  g.alpha = alpha; g.beta = beta;
  return run_gemm(ctx, g);
}

// update_renv!(env, A0, AR) (src/mps_base.jl:193-199): env(chiA, chiL0) = AR(chiA, drest) * A0(chiL0, drest)'
int op_update_renv(mpsb_ctx* ctx, const cd* A0, const cd* AR, cd* env, int chiA, int chiL0, int drest) {
  Gemm g;
  g.M = chiA; g.N = chiL0; g.K = drest;
  g.A = AR; g.a_m = 1; g.a_k = chiA;
  g.B = A0; g.b_k = chiL0; g.b_n = 1; g.conjB = true;
  g.C = env; g.c_m = 1; g.c_n = chiA;
  return run_gemm(ctx, g);
}

// update_lenv!(env, A0, AL) (src/mps_base.jl:275-281) and update_lenv_nc (:319-325):
// env(chiR0, y) = A0(lead, chiR0)' * AL(lead, y)   (.' when !conj)
int op_update_lenv(mpsb_ctx* ctx, const cd* A0, const cd* AL, cd* env, int lead, int chiR0, int y, bool conj) {
  Gemm g;
  g.M = chiR0; g.N = y; g.K = lead;
  g.A = A0; g.a_m = lead; g.a_k = 1; g.conjA = conj;
  g.B = AL; g.b_k = 1; g.b_n = lead;
  g.C = env; g.c_m = 1; g.c_n = chiR0;
  return run_gemm(ctx, g);
}

// QR through the context's workspace; a reallocated QR or split-K scratch (the blocked QR's
// trailing GEMMs may split K) invalidates captured graphs
int run_qr(mpsb_ctx* ctx, const QrProblem& p0) {
  QrProblem p = p0;
  int loops = 1;
  if (ctx->batch > 1 && p.batch == 1) {
    p.x_b = ctx->stride_of(p.X);
    p.q_b = ctx->stride_of(p.Q);
    p.r_b = p.R ? ctx->stride_of(p.R) : 0;
    if (qr_batch_supported(p.m, p.n)) p.batch = ctx->batch;
    else loops = ctx->batch;   // shapes beyond one cluster: one copy after the other
  }
  void* before = ctx->ws.qr.p;
  void* before_sk = ctx->ws.splitk.p;
  void* before_side = ctx->ws.qr_side_ws ? ctx->ws.qr_side_ws->splitk.p : nullptr;
  int st = MPSB_OK;
  for (int b = 0; b < loops && st == MPSB_OK; ++b) {
    QrProblem q = p;
    if (loops > 1) {
      q.X += b * p.x_b;
      q.Q += b * p.q_b;
      if (q.R) q.R += b * p.r_b;
    }
    count_launch(&ctx->ws);
    st = qr_launch(q, &ctx->ws, ctx->stream);
  }
  void* after_side = ctx->ws.qr_side_ws ? ctx->ws.qr_side_ws->splitk.p : nullptr;
  if (ctx->ws.qr.p != before || ctx->ws.splitk.p != before_sk || after_side != before_side) ctx->ws_generation++;
  return st;
}

// leftorth! / leftorth (src/orthonormalisation.jl:150-171): Q of reshape(A, Dl*d, Dr), in place
int op_orth_left(mpsb_ctx* ctx, cd* A, int Dl, int d, int Dr, cd* R) {
  QrProblem p;
  p.m = Dl * d; p.n = Dr;
  p.X = A; p.x_r = 1; p.x_c = (int64_t)Dl * d;
  p.Q = A; p.q_r = 1; p.q_c = (int64_t)Dl * d;
  if (R) { p.R = R; p.r_r = 1; p.r_c = Dr; }
  p.err = ctx->err();
  return run_qr(ctx, p);
}

// rightorth! (src/orthonormalisation.jl:227-234): QR of the non-conjugate transpose
// reshape(A, Dl, d*Dr).' and A = reshape(Q.', Dl, d, Dr), in place
int op_orth_right(mpsb_ctx* ctx, cd* A, int Dl, int d, int Dr) {
  QrProblem p;
  p.m = d * Dr; p.n = Dl;
  p.X = A; p.x_r = Dl; p.x_c = 1;
  p.Q = A; p.q_r = Dl; p.q_c = 1;
  p.err = ctx->err();
  return run_qr(ctx, p);
}

// ------------------------------------------------------------------------------------
static int same_dims(const mpsb_mps* a, const mpsb_mps* b) {
  return a && b && a->na == b->na && a->d == b->d && a->dims == b->dims;
}

int set_boundary(mpsb_ctx* ctx, cd* p, cd v) {
  count_launch(&ctx->ws);
  if (ctx->batch > 1) return set_value_strided(p, ctx->stride_of(p), ctx->batch, v, ctx->stream);
  return set_value(p, v, ctx->stream);
}

struct SweepScratch {
  cd* AOR; cd* AOL; cd* P[8];
};

static int sweep_scratch(mpsb_ctx* ctx, const mpsb_mps* A0, const mpsb_mpo* H, int nplain, SweepScratch& s) {
  int64_t maxAOR = 1, maxAOL = 1, maxSite = 1;
  const int d = A0->d;
  for (int k = 0; k < A0->na; ++k) {
    int64_t Dl = A0->dims[k], Dr = A0->dims[k + 1];
    if (H) {
      maxAOR = std::max<int64_t>(maxAOR, Dl * H->w[k] * d * Dr);
      maxAOL = std::max<int64_t>(maxAOL, Dl * d * Dr * H->w[k + 1]);
    }
    maxSite = std::max<int64_t>(maxSite, Dl * d * Dr);
  }
  s.AOR = s.AOL = nullptr;
  if (H) {
    MPSB_TRY(ensure_slot(ctx, SLOT_AOR, maxAOR * sizeof(cd), &s.AOR));
    MPSB_TRY(ensure_slot(ctx, SLOT_AOL, maxAOL * sizeof(cd), &s.AOL));
  }
  if (nplain > 8) return MPSB_ERR_UNSUPPORTED;
  cd* base = nullptr;
  if (nplain > 0) MPSB_TRY(ensure_slot(ctx, SLOT_P0, (size_t)nplain * maxSite * sizeof(cd), &base));
  for (int i = 0; i < nplain; ++i) s.P[i] = base + (int64_t)i * maxSite;
  return MPSB_OK;
}

static int sum_var_check(const mpsb_mps* A0, mpsb_env* const* env, const mpsb_env* envop, const mpsb_mps* Ain,
                         int numv, const mpsb_mps* const* A, const mpsb_mpo* H) {
  const int np = numv - 1;
  if (!same_dims(A0, Ain)) return MPSB_ERR_DIMENSION;
  for (int l = 0; l < numv; ++l)
    if (!same_dims(A0, A[l])) return MPSB_ERR_DIMENSION;
  for (int l = 0; l < np; ++l)
    if (!env || !env[l] || env[l]->three || env[l]->na != A0->na) return MPSB_ERR_DIMENSION;
  if (!envop->three || envop->na != A0->na || H->na != A0->na || H->d != A0->d) return MPSB_ERR_DIMENSION;
  for (int k = 0; k <= A0->na; ++k) {
    if (envop->d1[k] != A0->dims[k] || envop->d2[k] != A0->dims[k] || envop->w[k] != H->w[k]) return MPSB_ERR_DIMENSION;
    for (int l = 0; l < np; ++l)
      if (env[l]->d1[k] != A0->dims[k] || env[l]->d2[k] != A0->dims[k]) return MPSB_ERR_DIMENSION;
  }
  return MPSB_OK;
}

// Environment initialisation of a sum stage: left environments (L->R, for an R->L sweep) when
// !right, right environments (R->L) when right, from the bra Ain and the terms A (the last one
// through H), every chain advanced site by site in the order the previous stage finalises its
// sites.  `wait`, when given, holds one event per site that is waited on before site k is read.
static int sum_var_init(mpsb_ctx* ctx, bool right, mpsb_env* const* env, mpsb_env* envop, const mpsb_mps* Ain,
                        const cd* coef, int numv, const mpsb_mps* const* A, const mpsb_mpo* H, const SweepScratch& s,
                        const cudaEvent_t* wait) {
  const int np = numv - 1, na = Ain->na, d = Ain->d;
  const mpsb_mps* AH = A[np];
  auto D = [&](int k) { return (int)Ain->dims[k]; };
  auto W = [&](int k) { return (int)H->w[k]; };
  if (!right) {
    for (int l = 0; l < np; ++l) {
      MPSB_TRY(set_boundary(ctx, env[l]->entry(0), ONE));
      MPSB_TRY(set_boundary(ctx, env[l]->entry(na), coef[l]));
    }
    MPSB_TRY(set_boundary(ctx, envop->entry(0), ONE));
    MPSB_TRY(set_boundary(ctx, envop->entry(na), coef[np]));
    for (int k = 0; k < na - 1; ++k) {
      if (wait) MPSB_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, wait[k], 0));
      for (int l = 0; l < np; ++l) {
        MPSB_TRY(op_L2_A3(ctx, env[l]->entry(k), A[l]->site(k), s.P[l], D(k), D(k), d * D(k + 1), ONE, ZERO, false));
        MPSB_TRY(op_update_lenv(ctx, Ain->site(k), s.P[l], env[l]->entry(k + 1), D(k) * d, D(k + 1), D(k + 1), true));
      }
      MPSB_TRY(op_prod_AOL(ctx, AH->site(k), H->site(k), envop->entry(k), s.AOL, D(k), d, D(k + 1), W(k), W(k + 1), D(k)));
      MPSB_TRY(op_update_le(ctx, Ain->site(k), s.AOL, envop->entry(k + 1), D(k), d, D(k + 1), W(k + 1), D(k + 1)));
    }
  } else {
    for (int l = 0; l < np; ++l) {
      MPSB_TRY(set_boundary(ctx, env[l]->entry(na), ONE));
      MPSB_TRY(set_boundary(ctx, env[l]->entry(0), coef[l]));
    }
    MPSB_TRY(set_boundary(ctx, envop->entry(na), ONE));
    MPSB_TRY(set_boundary(ctx, envop->entry(0), coef[np]));
    for (int k = na - 1; k >= 1; --k) {
      if (wait) MPSB_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, wait[k], 0));
      for (int l = 0; l < np; ++l) {
        MPSB_TRY(op_A3_R2(ctx, A[l]->site(k), env[l]->entry(k + 1), s.P[l], D(k) * d, D(k + 1), D(k + 1), ONE, ZERO));
        MPSB_TRY(op_update_renv(ctx, Ain->site(k), s.P[l], env[l]->entry(k), D(k), D(k), d * D(k + 1)));
      }
      MPSB_TRY(op_prod_AOR(ctx, AH->site(k), H->site(k), envop->entry(k + 1), s.AOR, D(k), d, D(k + 1), W(k), W(k + 1), D(k + 1)));
      MPSB_TRY(op_update_re(ctx, Ain->site(k), s.AOR, envop->entry(k), D(k), W(k), d, D(k + 1), D(k)));
    }
  }
  return MPSB_OK;
}

// The half sweep of a sum stage (R->L when !right, L->R when right) writing A0 site by site;
// `rec`, when given, gets one event per site recorded as soon as that site of A0 is final.
static int sum_var_sweep(mpsb_ctx* ctx, bool right, mpsb_mps* A0, mpsb_env* const* env, mpsb_env* envop, int numv,
                         const mpsb_mps* const* A, const mpsb_mpo* H, const SweepScratch& s, const cudaEvent_t* rec) {
  const int np = numv - 1, na = A0->na, d = A0->d;
  const mpsb_mps* AH = A[np];
  auto D = [&](int k) { return (int)A0->dims[k]; };
  auto W = [&](int k) { return (int)H->w[k]; };
  auto final_site = [&](int k) -> int {
    if (rec) MPSB_CUDA_TRY(cudaEventRecord(rec[k], ctx->stream));
    return MPSB_OK;
  };
  if (!right) {
    for (int k = na - 1; k >= 0; --k) {
      cd* out = A0->site(k);
      for (int l = 0; l < np; ++l) {
        MPSB_TRY(op_A3_R2(ctx, A[l]->site(k), env[l]->entry(k + 1), s.P[l], D(k) * d, D(k + 1), D(k + 1), ONE, ZERO));
        MPSB_TRY(op_L2_A3(ctx, env[l]->entry(k), s.P[l], out, D(k), D(k), d * D(k + 1), ONE, l ? ONE : ZERO, false));
      }
      MPSB_TRY(op_prod_AOR(ctx, AH->site(k), H->site(k), envop->entry(k + 1), s.AOR, D(k), d, D(k + 1), W(k), W(k + 1), D(k + 1)));
      MPSB_TRY(op_prod_LR_3_4(ctx, envop->entry(k), s.AOR, out, D(k), W(k), D(k), d, D(k + 1), ONE, np ? ONE : ZERO));
      if (k == 0) {
        MPSB_TRY(final_site(0));
        break;
      }
      MPSB_TRY(op_orth_right(ctx, out, D(k), d, D(k + 1)));
      MPSB_TRY(final_site(k));
      for (int l = 0; l < np; ++l)
        MPSB_TRY(op_update_renv(ctx, out, s.P[l], env[l]->entry(k), D(k), D(k), d * D(k + 1)));
      MPSB_TRY(op_update_re(ctx, out, s.AOR, envop->entry(k), D(k), W(k), d, D(k + 1), D(k)));
    }
  } else {
    for (int k = 0; k < na; ++k) {
      cd* out = A0->site(k);
      for (int l = 0; l < np; ++l) {
        MPSB_TRY(op_L2_A3(ctx, env[l]->entry(k), A[l]->site(k), s.P[l], D(k), D(k), d * D(k + 1), ONE, ZERO, false));
        MPSB_TRY(op_A3_R2(ctx, s.P[l], env[l]->entry(k + 1), out, D(k) * d, D(k + 1), D(k + 1), ONE, l ? ONE : ZERO));
      }
      MPSB_TRY(op_prod_AOL(ctx, AH->site(k), H->site(k), envop->entry(k), s.AOL, D(k), d, D(k + 1), W(k), W(k + 1), D(k)));
      MPSB_TRY(op_prod_LR_4_3(ctx, s.AOL, envop->entry(k + 1), out, D(k), d, D(k + 1), W(k + 1), D(k + 1), ONE, np ? ONE : ZERO));
      if (k == na - 1) {
        MPSB_TRY(final_site(k));
        break;
      }
      MPSB_TRY(op_orth_left(ctx, out, D(k), d, D(k + 1), nullptr));
      MPSB_TRY(final_site(k));
      for (int l = 0; l < np; ++l)
        MPSB_TRY(op_update_lenv(ctx, out, s.P[l], env[l]->entry(k + 1), D(k) * d, D(k + 1), D(k + 1), true));
      MPSB_TRY(op_update_le(ctx, out, s.AOL, envop->entry(k + 1), D(k), d, D(k + 1), W(k + 1), D(k + 1)));
    }
  }
  return MPSB_OK;
}

// compress_sum_var_apply_H_left! (src/compression.jl:889-944) when !right,
// compress_sum_var_apply_H_right! (src/compression.jl:1007-1063) when right.
// numv == 1 with coef {1} is compress_var_apply_H_left! (src/compression.jl:321-347).
int compress_sum_var_apply_H(mpsb_ctx* ctx, bool right, mpsb_mps* A0, mpsb_env* const* env, mpsb_env* envop,
                             const mpsb_mps* Ain, const cd* coef, int numv, const mpsb_mps* const* A,
                             const mpsb_mpo* H) {
  if (!ctx || !A0 || !envop || !Ain || !coef || !A || !H || numv < 1) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(sum_var_check(A0, env, envop, Ain, numv, A, H));
  SplitScope scope(ctx);
  int B;
  bool batched;
  MPSB_TRY(call_batch({A0, Ain}, {envop}, &B, &batched));
  for (int l = 0; l < numv; ++l)
    if (A[l]->batch != B || (l < numv - 1 && env[l]->batch != B)) return MPSB_ERR_DIMENSION;
  BatchScope bscope(ctx, B, batched);
  SweepScratch s;
  MPSB_TRY(sweep_scratch(ctx, A0, H, numv - 1, s));
  MPSB_TRY(sum_var_init(ctx, right, env, envop, Ain, coef, numv, A, H, s, nullptr));
  return sum_var_sweep(ctx, right, A0, env, envop, numv, A, H, s, nullptr);
}

int compress_var_apply_H_left(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain, const mpsb_mps* A,
                              const mpsb_mpo* H) {
  const mpsb_mps* terms[1] = {A};
  cd c1[1] = {ONE};
  return compress_sum_var_apply_H(ctx, false, A0, nullptr, envop, Ain, c1, 1, terms, H);
}

// Run `body` (a fixed sequence of launches on the context's streams) through the context's graph
// cache: the first call runs eagerly and sizes every scratch buffer, the second captures the
// launches into a CUDA graph, later calls replay it; a reallocated scratch buffer (generation
// counter) sends the key back to eager execution.  With graphs off, the body runs eagerly.
static int run_cached(mpsb_ctx* ctx, const std::vector<int64_t>& key, const std::function<int()>& body) {
  if (!ctx->graphs) return body();
  auto& ent = ctx->graphs_cache[key];
  if (ent.exec && ent.generation == ctx->ws_generation) {
    ctx->ws.launches += ent.launches;
    MPSB_CUDA_TRY(cudaGraphLaunch(ent.exec, ctx->stream));
    return MPSB_OK;
  }
  if (ent.exec) {
    cudaGraphExecDestroy(ent.exec);
    ent.exec = nullptr;
    ent.seen = 0;
  }
  if (ent.seen == 0) {  // eager first call sizes every scratch buffer
    ent.seen = 1;
    return body();
  }
  const int64_t gen0 = ctx->ws_generation;
  const int64_t l0 = ctx->ws.launches + ctx->ws_side.launches;
  ctx->ws.capturing = ctx->ws_side.capturing = true;
  MPSB_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int st = body();
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
  ctx->ws.capturing = ctx->ws_side.capturing = false;
  if (st != MPSB_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (ce != cudaSuccess) {
    set_last_error(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
    return MPSB_ERR_CUDA;
  }
  cudaGraphExec_t exec = nullptr;
  ce = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    set_last_error(ce, "cudaGraphInstantiate", __FILE__, __LINE__);
    return MPSB_ERR_CUDA;
  }
  ent.exec = exec;
  ent.generation = gen0;
  ent.launches = ctx->ws.launches + ctx->ws_side.launches - l0;
  MPSB_CUDA_TRY(cudaGraphLaunch(exec, ctx->stream));
  return MPSB_OK;
}

static int compress_var_apply_H_body(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain,
                                     const mpsb_mps* A, const mpsb_mpo* H, int maxsweeps);

// compress_var_apply_H! (src/compression.jl:217-258): maxsweeps R->L / L->R sweep pairs
int compress_var_apply_H(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain, const mpsb_mps* A,
                         const mpsb_mpo* H, int maxsweeps) {
  if (!ctx || !A0 || !envop || !Ain || !A || !H || maxsweeps < 0) return MPSB_ERR_INVALID_ARG;
  if (!same_dims(A0, Ain) || !same_dims(A0, A) || !envop->three || H->na != A0->na) return MPSB_ERR_DIMENSION;
  SplitScope scope(ctx);
  int B;
  bool batched;
  MPSB_TRY(call_batch({A0, Ain, A}, {envop}, &B, &batched));
  BatchScope bscope(ctx, B, batched);
  std::vector<int64_t> key = {2, ctx->split_slices, ctx->split_min_tiles, (int64_t)ctx->split_min_flops, B, maxsweeps, A0->serial, envop->serial,
                              Ain->serial, A->serial, H->serial};
  return run_cached(ctx, key, [&]() { return compress_var_apply_H_body(ctx, A0, envop, Ain, A, H, maxsweeps); });
}

static int compress_var_apply_H_body(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain,
                                     const mpsb_mps* A, const mpsb_mpo* H, int maxsweeps) {
  const int na = A0->na, d = A0->d;
  for (int k = 0; k <= na; ++k)
    if (envop->d1[k] != A0->dims[k] || envop->d2[k] != A0->dims[k] || envop->w[k] != H->w[k]) return MPSB_ERR_DIMENSION;
  SweepScratch s;
  MPSB_TRY(sweep_scratch(ctx, A0, H, 0, s));
  auto D = [&](int k) { return (int)A0->dims[k]; };
  auto W = [&](int k) { return (int)H->w[k]; };
  MPSB_TRY(set_boundary(ctx, envop->entry(0), ONE));
  for (int k = 0; k < na - 1; ++k) {
    MPSB_TRY(op_prod_AOL(ctx, A->site(k), H->site(k), envop->entry(k), s.AOL, D(k), d, D(k + 1), W(k), W(k + 1), D(k)));
    MPSB_TRY(op_update_le(ctx, Ain->site(k), s.AOL, envop->entry(k + 1), D(k), d, D(k + 1), W(k + 1), D(k + 1)));
  }
  MPSB_TRY(set_boundary(ctx, envop->entry(na), ONE));
  for (int sw = 0; sw < maxsweeps; ++sw) {
    for (int k = na - 1; k >= 1; --k) {
      MPSB_TRY(op_prod_AOR(ctx, A->site(k), H->site(k), envop->entry(k + 1), s.AOR, D(k), d, D(k + 1), W(k), W(k + 1), D(k + 1)));
      MPSB_TRY(op_prod_LR_3_4(ctx, envop->entry(k), s.AOR, A0->site(k), D(k), W(k), D(k), d, D(k + 1), ONE, ZERO));
      MPSB_TRY(op_orth_right(ctx, A0->site(k), D(k), d, D(k + 1)));
      MPSB_TRY(op_update_re(ctx, A0->site(k), s.AOR, envop->entry(k), D(k), W(k), d, D(k + 1), D(k)));
    }
    for (int k = 0; k < na; ++k) {
      MPSB_TRY(op_prod_AOL(ctx, A->site(k), H->site(k), envop->entry(k), s.AOL, D(k), d, D(k + 1), W(k), W(k + 1), D(k)));
      MPSB_TRY(op_prod_LR_4_3(ctx, s.AOL, envop->entry(k + 1), A0->site(k), D(k), d, D(k + 1), W(k + 1), D(k + 1), ONE, ZERO));
      if (k == na - 1) break;
      MPSB_TRY(op_orth_left(ctx, A0->site(k), D(k), d, D(k + 1), nullptr));
      MPSB_TRY(op_update_le(ctx, A0->site(k), s.AOL, envop->entry(k + 1), D(k), d, D(k + 1), W(k + 1), D(k + 1)));
    }
  }
  return MPSB_OK;
}

// compress_sum_var_apply_H! (src/compression.jl:805-887) when H is given -- the last term is
// H * A[numv-1] with its coefficient at envop's right boundary -- and compress_sum_var
// (src/compression.jl:496-565) when H is null (every term plain): maxsweeps R->L / L->R sweep
// pairs of the variational compression of the weighted sum, then the last site.  A0 is the
// guess (the bra of the initial left environments) and is overwritten with the result; it
// must not be one of the terms.  The plain-term environments live in context scratch.
int compress_sum_var_full(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const cd* coef, int numv,
                          const mpsb_mps* const* A, const mpsb_mpo* H, int maxsweeps) {
  if (!ctx || !A0 || !coef || !A || numv < 1 || maxsweeps < 0) return MPSB_ERR_INVALID_ARG;
  const bool hasH = H != nullptr;
  SplitScope scope(ctx);
  int B;
  bool batched;
  MPSB_TRY(call_batch({A0}, {hasH ? envop : nullptr}, &B, &batched));
  for (int l = 0; l < numv; ++l)
    if (A[l] && A[l]->batch != B) return MPSB_ERR_DIMENSION;
  BatchScope bscope(ctx, B, batched);
  if (hasH && !envop) return MPSB_ERR_INVALID_ARG;
  const int np = hasH ? numv - 1 : numv;
  if (np < 1) {   // the reference indexes the first plain term unconditionally
    set_last_message("compress_sum_var: at least one plain term is required");
    return MPSB_ERR_INVALID_ARG;
  }
  if (np > 8) return MPSB_ERR_UNSUPPORTED;
  for (int l = 0; l < numv; ++l) {
    if (!A[l] || !same_dims(A0, A[l])) return MPSB_ERR_DIMENSION;
    if (A[l] == A0 || A[l]->slab == A0->slab) {
      set_last_message("compress_sum_var: the output MPS must not be one of the terms");
      return MPSB_ERR_INVALID_ARG;
    }
  }
  const int na = A0->na, d = A0->d;
  if (hasH) {
    if (!envop->three || envop->na != na || H->na != na || H->d != d) return MPSB_ERR_DIMENSION;
    for (int k = 0; k <= na; ++k)
      if (envop->d1[k] != A0->dims[k] || envop->d2[k] != A0->dims[k] || envop->w[k] != H->w[k])
        return MPSB_ERR_DIMENSION;
  }
  SweepScratch s;
  MPSB_TRY(sweep_scratch(ctx, A0, H, np, s));
  auto D = [&](int k) { return (int)A0->dims[k]; };
  auto W = [&](int k) { return (int)H->w[k]; };
  std::vector<int64_t> eoff(na + 1);
  int64_t etot = 0;
  for (int k = 0; k <= na; ++k) {
    eoff[k] = etot;
    etot += A0->dims[k] * A0->dims[k];
  }
  cd* ebase = nullptr;
  MPSB_TRY(ensure_slot(ctx, SLOT_SUMENV, (size_t)np * etot * sizeof(cd), &ebase));
  auto E = [&](int l, int k) { return ebase + (int64_t)l * etot + eoff[k]; };
  const mpsb_mps* AH = hasH ? A[np] : nullptr;

  // ---- left environments with A0 as the bra
  for (int l = 0; l < np; ++l) {
    MPSB_TRY(set_boundary(ctx, E(l, 0), ONE));
    for (int k = 0; k < na - 1; ++k) {
      MPSB_TRY(op_L2_A3(ctx, E(l, k), A[l]->site(k), s.P[l], D(k), D(k), d * D(k + 1), ONE, ZERO, false));
      MPSB_TRY(op_update_lenv(ctx, A0->site(k), s.P[l], E(l, k + 1), D(k) * d, D(k + 1), D(k + 1), true));
    }
    MPSB_TRY(set_boundary(ctx, E(l, na), coef[l]));
  }
  if (hasH) {
    MPSB_TRY(set_boundary(ctx, envop->entry(0), ONE));
    for (int k = 0; k < na - 1; ++k) {
      MPSB_TRY(op_prod_AOL(ctx, AH->site(k), H->site(k), envop->entry(k), s.AOL, D(k), d, D(k + 1), W(k), W(k + 1), D(k)));
      MPSB_TRY(op_update_le(ctx, A0->site(k), s.AOL, envop->entry(k + 1), D(k), d, D(k + 1), W(k + 1), D(k + 1)));
    }
    MPSB_TRY(set_boundary(ctx, envop->entry(na), coef[np]));
  }
  // site k of the L->R direction: plain terms, then the H term, accumulated into A0[k]
  auto site_lr = [&](int k) -> int {
    cd* out = A0->site(k);
    for (int l = 0; l < np; ++l) {
      MPSB_TRY(op_L2_A3(ctx, E(l, k), A[l]->site(k), s.P[l], D(k), D(k), d * D(k + 1), ONE, ZERO, false));
      MPSB_TRY(op_A3_R2(ctx, s.P[l], E(l, k + 1), out, D(k) * d, D(k + 1), D(k + 1), ONE, l ? ONE : ZERO));
    }
    if (hasH) {
      MPSB_TRY(op_prod_AOL(ctx, AH->site(k), H->site(k), envop->entry(k), s.AOL, D(k), d, D(k + 1), W(k), W(k + 1), D(k)));
      MPSB_TRY(op_prod_LR_4_3(ctx, s.AOL, envop->entry(k + 1), out, D(k), d, D(k + 1), W(k + 1), D(k + 1), ONE, ONE));
    }
    return MPSB_OK;
  };
  for (int sw = 0; sw < maxsweeps; ++sw) {
    for (int k = na - 1; k >= 1; --k) {   // sweep left
      cd* out = A0->site(k);
      for (int l = 0; l < np; ++l) {
        MPSB_TRY(op_A3_R2(ctx, A[l]->site(k), E(l, k + 1), s.P[l], D(k) * d, D(k + 1), D(k + 1), ONE, ZERO));
        MPSB_TRY(op_L2_A3(ctx, E(l, k), s.P[l], out, D(k), D(k), d * D(k + 1), ONE, l ? ONE : ZERO, false));
      }
      if (hasH) {
        MPSB_TRY(op_prod_AOR(ctx, AH->site(k), H->site(k), envop->entry(k + 1), s.AOR, D(k), d, D(k + 1), W(k), W(k + 1), D(k + 1)));
        MPSB_TRY(op_prod_LR_3_4(ctx, envop->entry(k), s.AOR, out, D(k), W(k), D(k), d, D(k + 1), ONE, ONE));
      }
      MPSB_TRY(op_orth_right(ctx, out, D(k), d, D(k + 1)));
      for (int l = 0; l < np; ++l)
        MPSB_TRY(op_update_renv(ctx, out, s.P[l], E(l, k), D(k), D(k), d * D(k + 1)));
      if (hasH) MPSB_TRY(op_update_re(ctx, out, s.AOR, envop->entry(k), D(k), W(k), d, D(k + 1), D(k)));
    }
    for (int k = 0; k < na - 1; ++k) {   // sweep right
      MPSB_TRY(site_lr(k));
      cd* out = A0->site(k);
      MPSB_TRY(op_orth_left(ctx, out, D(k), d, D(k + 1), nullptr));
      for (int l = 0; l < np; ++l)
        MPSB_TRY(op_update_lenv(ctx, out, s.P[l], E(l, k + 1), D(k) * d, D(k + 1), D(k + 1), true));
      if (hasH) MPSB_TRY(op_update_le(ctx, out, s.AOL, envop->entry(k + 1), D(k), d, D(k + 1), W(k + 1), D(k + 1)));
    }
  }
  return site_lr(na - 1);
}

// RK4stp_apply_H_half! (src/timeevolution.jl:178-196), one stage after the other
static int rk4_body_serial(mpsb_ctx* ctx, double dt, const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3,
                           mpsb_mps* psi0, mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2, mpsb_mps* psi3,
                           mpsb_env* env1, mpsb_env* env2, mpsb_env* env3, mpsb_env* envop) {
  MPSB_TRY(compress_var_apply_H_left(ctx, psi1, envop, psi, psi, H1));
  {
    mpsb_env* e[1] = {env1};
    const mpsb_mps* t[2] = {psi, psi1};
    cd c[2] = {ONE, cmk(dt / 2, 0.0)};
    MPSB_TRY(compress_sum_var_apply_H(ctx, true, psi2, e, envop, psi1, c, 2, t, H2));
  }
  {
    mpsb_env* e[1] = {env1};
    const mpsb_mps* t[2] = {psi, psi2};
    cd c[2] = {ONE, cmk(dt, 0.0)};
    MPSB_TRY(compress_sum_var_apply_H(ctx, false, psi3, e, envop, psi2, c, 2, t, H2));
  }
  {
    mpsb_env* e[3] = {env1, env2, env3};
    const mpsb_mps* t[4] = {psi, psi1, psi2, psi3};
    cd c[4] = {cmk(-1.0 / 3, 0.0), cmk(1.0 / 3, 0.0), cmk(2.0 / 3, 0.0), cmk(1.0 / 3, 0.0)};
    MPSB_TRY(compress_sum_var_apply_H(ctx, true, psi0, e, envop, psi3, c, 4, t, H3));
  }
  return MPSB_OK;
}

// Scratch for any of the four stages (three plain terms, the widest of the three operators);
// slots only grow, so the pointers of the last call stay valid for all.
static int sweep_scratch_all(mpsb_ctx* ctx, const mpsb_mps* A0, const mpsb_mpo* H1, const mpsb_mpo* H2,
                             const mpsb_mpo* H3, SweepScratch& s) {
  MPSB_TRY(sweep_scratch(ctx, A0, H1, 3, s));
  MPSB_TRY(sweep_scratch(ctx, A0, H2, 3, s));
  return sweep_scratch(ctx, A0, H3, 3, s);
}

// While alive, work is issued on the context's second lane (stream `side`, workspace ws_side).
struct SideLane {
  mpsb_ctx* c;
  cudaStream_t saved;
  explicit SideLane(mpsb_ctx* ctx) : c(ctx), saved(ctx->stream) {
    c->stream = c->side;
    std::swap(c->ws, c->ws_side);
  }
  ~SideLane() {
    std::swap(c->ws, c->ws_side);
    c->stream = saved;
  }
};

static int ensure_events(mpsb_ctx* ctx, size_t n) {
  while (ctx->events.size() < n) {
    cudaEvent_t ev;
    MPSB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    ctx->events.push_back(ev);
  }
  return MPSB_OK;
}

// An environment stack shaped like `like` whose storage is a context scratch slot.
static int scratch_env(mpsb_ctx* ctx, Slot slot, const mpsb_env* like, mpsb_env& out) {
  out = *like;
  out.serial = 0;
  return ensure_slot(ctx, slot, (size_t)like->total * sizeof(cd), &out.slab);
}

// The same four stages with each stage's environment initialisation (which reads the previous
// stage's output site by site, in the order that stage finalises them) issued on the second
// lane, waiting per site, so it runs beside the previous stage's sweep -- in particular beside
// its QRs, which occupy one thread-block cluster.  Every computation is the one of the serial
// body, so the results are identical.  Stages 2 and 4 use an internal envop, stage 3 env2 and
// stage 4 an internal third plain-term environment, so that concurrent stages never share an
// environment buffer.
static int rk4_body_pipelined(mpsb_ctx* ctx, double dt, const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3,
                              mpsb_mps* psi0, mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2, mpsb_mps* psi3,
                              mpsb_env* env1, mpsb_env* env2, mpsb_env* env3, mpsb_env* envop) {
  const int na = psi->na;
  MPSB_TRY(ensure_events(ctx, (size_t)3 * na + 4));
  cudaEvent_t* ev = ctx->events.data();
  cudaEvent_t* site_ev[3] = {ev, ev + na, ev + 2 * na};
  cudaEvent_t done[3] = {ev[3 * na], ev[3 * na + 1], ev[3 * na + 2]};
  cudaEvent_t fork = ev[3 * na + 3];
  mpsb_env envopB, envX;
  MPSB_TRY(scratch_env(ctx, SLOT_PIPE_ENVOP, envop, envopB));
  MPSB_TRY(scratch_env(ctx, SLOT_PIPE_ENV, env1, envX));

  // stage descriptions: which half sweep, output, bra, terms, coefficients, operator, envs
  const cd c1[1] = {ONE};
  const cd c2[2] = {ONE, cmk(dt / 2, 0.0)};
  const cd c3[2] = {ONE, cmk(dt, 0.0)};
  const cd c4[4] = {cmk(-1.0 / 3, 0.0), cmk(1.0 / 3, 0.0), cmk(2.0 / 3, 0.0), cmk(1.0 / 3, 0.0)};
  const mpsb_mps* t1[1] = {psi};
  const mpsb_mps* t2[2] = {psi, psi1};
  const mpsb_mps* t3[2] = {psi, psi2};
  const mpsb_mps* t4[4] = {psi, psi1, psi2, psi3};
  mpsb_env* e2[1] = {env1};
  mpsb_env* e3[1] = {env2};
  mpsb_env* e4[3] = {env1, env3, &envX};
  struct Stage {
    bool right; mpsb_mps* A0; const mpsb_mps* Ain; const cd* coef; int numv; const mpsb_mps* const* A;
    const mpsb_mpo* H; mpsb_env* const* env; mpsb_env* envop;
  };
  const Stage st[4] = {{false, psi1, psi, c1, 1, t1, H1, nullptr, envop},
                       {true, psi2, psi1, c2, 2, t2, H2, e2, &envopB},
                       {false, psi3, psi2, c3, 2, t3, H2, e3, envop},
                       {true, psi0, psi3, c4, 4, t4, H3, e4, &envopB}};
  for (const Stage& g : st) MPSB_TRY(sum_var_check(g.A0, g.env, g.envop, g.Ain, g.numv, g.A, g.H));

  SweepScratch sm;   // main lane scratch, sized for every stage
  MPSB_TRY(sweep_scratch_all(ctx, psi, H1, H2, H3, sm));
  MPSB_CUDA_TRY(cudaEventRecord(fork, ctx->stream));
  MPSB_TRY(sum_var_init(ctx, st[0].right, st[0].env, st[0].envop, st[0].Ain, st[0].coef, st[0].numv, st[0].A, st[0].H, sm,
                        nullptr));
  for (int i = 0; i < 4; ++i) {
    const Stage& g = st[i];
    MPSB_TRY(sum_var_sweep(ctx, g.right, g.A0, g.env, g.envop, g.numv, g.A, g.H, sm, i < 3 ? site_ev[i] : nullptr));
    if (i == 3) break;
    const Stage& n = st[i + 1];
    {
      SideLane lane(ctx);
      if (i == 0) MPSB_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, fork, 0));
      SweepScratch ss;
      MPSB_TRY(sweep_scratch_all(ctx, psi, H1, H2, H3, ss));
      MPSB_TRY(sum_var_init(ctx, n.right, n.env, n.envop, n.Ain, n.coef, n.numv, n.A, n.H, ss, site_ev[i]));
      MPSB_CUDA_TRY(cudaEventRecord(done[i], ctx->stream));
    }
    MPSB_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, done[i], 0));
  }
  return MPSB_OK;
}

static int rk4_body(mpsb_ctx* ctx, double dt, const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3,
                    mpsb_mps* psi0, mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2, mpsb_mps* psi3, mpsb_env* env1,
                    mpsb_env* env2, mpsb_env* env3, mpsb_env* envop) {
  if (ctx->pipeline && ctx->side)
    return rk4_body_pipelined(ctx, dt, H1, H2, H3, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop);
  return rk4_body_serial(ctx, dt, H1, H2, H3, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop);
}

int rk4_step(mpsb_ctx* ctx, double dt, const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3, mpsb_mps* psi0,
             mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2, mpsb_mps* psi3, mpsb_env* env1, mpsb_env* env2,
             mpsb_env* env3, mpsb_env* envop) {
  if (!ctx || !H1 || !H2 || !H3 || !psi0 || !psi || !psi1 || !psi2 || !psi3 || !env1 || !env2 || !env3 || !envop)
    return MPSB_ERR_INVALID_ARG;
  SplitScope scope(ctx);
  int B;
  bool batched;
  MPSB_TRY(call_batch({psi0, psi, psi1, psi2, psi3}, {env1, env2, env3, envop}, &B, &batched));
  BatchScope bscope(ctx, B, batched);
  int64_t dtbits;
  std::memcpy(&dtbits, &dt, sizeof(dt));
  std::vector<int64_t> key = {1, ctx->pipeline ? 2 : 1, ctx->split_slices, ctx->split_min_tiles,
                               (int64_t)ctx->split_min_flops, B, dtbits,
                              H1->serial, H2->serial, H3->serial, psi0->serial, psi->serial, psi1->serial,
                              psi2->serial, psi3->serial, env1->serial, env2->serial, env3->serial, envop->serial};
  return run_cached(ctx, key, [&]() {
    return rk4_body(ctx, dt, H1, H2, H3, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop);
  });
}

}  // namespace mpsb
