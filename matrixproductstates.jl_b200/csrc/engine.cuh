// Handles and host-side sweep orchestration of the mpsb200 engine.
#pragma once
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "misc.cuh"
#include "workspace.cuh"

struct mpsb_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  mpsb::Workspace ws;
  // second lane of the RK4 step: the next stage's environment initialisation runs on `side`
  // with its own scratch and split-K workspace (swapped into `ws`/`stream` while it issues)
  cudaStream_t side = nullptr;
  mpsb::Workspace ws_side;
  std::vector<cudaEvent_t> events;   // per-site / fork / join events, created on first use
  bool pipeline = true;
  bool graphs = true;
  // contraction precision of the sweeps: 0 = FP64 (DMMA); 3..7 = int8-sliced tensor-core GEMM
  // with that many slices per operand, used for GEMMs of at least split_min_tiles output tiles
  int split_slices = 0;
  int split_min_tiles = 64;
  double split_min_flops = 16777216.0;   // batched calls: one copy's 8 M N K at least this
  bool split_on = false;       // set while a sweep entry point issues its contractions
  // batched calls: every MPS / environment handle of the call holds `batch` copies of the same
  // shape back to back, and each kernel runs all copies at once.  The registry maps the base of
  // every batched slab (handles and scratch slots) to its end and its copy stride (elements);
  // a pointer outside every registered slab (an MPO) is shared by all copies.
  int batch = 1;
  mpsb::DevBuf vec;   // per-copy results of batched calls (norms)
  struct Slab {
    uintptr_t end;
    int64_t stride;
  };
  std::map<uintptr_t, Slab> slabs;
  int64_t stride_of(const void* p) const {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    auto it = slabs.upper_bound(a);
    if (it == slabs.begin()) return 0;
    --it;
    return a < it->second.end ? it->second.stride : 0;
  }
  int64_t ws_generation = 0;   // bumped whenever a scratch buffer is reallocated
  double* d_scalars = nullptr; // small device scratch for norms (64 doubles)
  double* h_scalars = nullptr; // pinned host mirror
  // device error word (inside d_scalars[63]): kernels whose bounded waits run out set a bit
  // (bit 0: the QR cluster's exchanges, bit 1: the sliced GEMM's pipeline)
  int* err() const { return reinterpret_cast<int*>(d_scalars + 63); }
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    int64_t generation = -1;
    int64_t launches = 0;  // kernel nodes recorded at capture, added on every replay
    int seen = 0;
  };
  std::map<std::vector<int64_t>, GraphEntry> graphs_cache;
  std::vector<mpsb::Workspace::TimedLaunch> prof_events;   // see mpsb_ctx_set_profiling
};

struct mpsb_mps {
  mpsb_ctx* ctx = nullptr;
  int64_t serial = 0;
  int batch = 1;          // copies in the slab (copy stride = total)
  bool batched = false;   // a batch handle or a view of one copy: calls run in batched mode
  bool owns = true;       // false for a view (the slab belongs to the batch handle)
  int na = 0, d = 0;
  std::vector<int64_t> dims;   // na+1
  std::vector<int64_t> off;    // element offset of each site
  mpsb::cd* slab = nullptr;
  int64_t total = 0;
  mpsb::cd* site(int s) const { return slab + off[s]; }
  int64_t site_elems(int s) const { return dims[s] * d * dims[s + 1]; }
};

struct mpsb_mpo {
  mpsb_ctx* ctx = nullptr;
  int64_t serial = 0;
  int na = 0, d = 0;
  std::vector<int64_t> w;      // na+1
  std::vector<int64_t> off;
  mpsb::cd* slab = nullptr;
  int64_t total = 0;
  mpsb::cd* site(int s) const { return slab + off[s]; }
  int64_t site_elems(int s) const { return w[s] * d * w[s + 1] * d; }
};

struct mpsb_env {
  mpsb_ctx* ctx = nullptr;
  int64_t serial = 0;
  int batch = 1;          // copies in the slab (copy stride = total)
  bool batched = false;
  int na = 0;
  bool three = false;
  std::vector<int64_t> d1, d2, w;  // na+1 each (w all 1 for 2-index)
  std::vector<int64_t> off;
  mpsb::cd* slab = nullptr;
  int64_t total = 0;
  mpsb::cd* entry(int e) const { return slab + off[e]; }
  int64_t entry_elems(int e) const { return d1[e] * w[e] * d2[e]; }
};

namespace mpsb {

// named scratch slots in Workspace::named
enum Slot {
  SLOT_T = 0, SLOT_AOR, SLOT_G1, SLOT_AOL, SLOT_P0, SLOT_P1, SLOT_P2, SLOT_ENV0, SLOT_ENV1,
  SLOT_MISC, SLOT_SUMENV, SLOT_GSENV, SLOT_GSVEC, SLOT_PIPE_ENVOP, SLOT_PIPE_ENV, SLOT_COUNT
};

int ensure_slot(mpsb_ctx* ctx, Slot s, size_t bytes, cd** out);

// ---- single contractions (device pointers, dims explicit); alpha/beta accumulate into out
int op_prod_AOR(mpsb_ctx* ctx, const cd* A, const cd* O, const cd* R, cd* AOR, int chiL, int d, int chiR,
                int wL, int wR, int chiR0);
int op_prod_AOL(mpsb_ctx* ctx, const cd* A, const cd* O, const cd* L, cd* AOL, int chiL, int d, int chiR,
                int wL, int wR, int chiL0);
int op_prod_LR_3_4(mpsb_ctx* ctx, const cd* L, const cd* AOR, cd* A0, int chiL, int wL, int chiL0, int d,
                   int chiR0, cd alpha, cd beta);
int op_prod_LR_4_3(mpsb_ctx* ctx, const cd* AOL, const cd* R, cd* A0, int chiL0, int d, int chiR, int wR,
                   int chiR0, cd alpha, cd beta);
int op_update_re(mpsb_ctx* ctx, const cd* A0, const cd* AOR, cd* env, int chiL, int wL, int d, int chiR0,
                 int chiL0);
int op_update_le(mpsb_ctx* ctx, const cd* A0, const cd* AOL, cd* env, int chiL0, int d, int chiR, int wR,
                 int chiR0);
// 2-index env products
int op_L2_A3(mpsb_ctx* ctx, const cd* L, const cd* A, cd* out, int x, int chiL, int rest, cd alpha, cd beta,
             bool transL);
int op_A3_R2(mpsb_ctx* ctx, const cd* A, const cd* R, cd* out, int lead, int chiR, int y, cd alpha, cd beta);
int op_update_renv(mpsb_ctx* ctx, const cd* A0, const cd* AR, cd* env, int chiA, int chiL0, int drest);
int op_update_lenv(mpsb_ctx* ctx, const cd* A0, const cd* AL, cd* env, int lead, int chiR0, int y, bool conj);
// QR of a site: left (reshape(A, Dl*d, Dr)) or right (transpose of reshape(A, Dl, d*Dr))
int run_qr(mpsb_ctx* ctx, const QrProblem& p);
int run_gemm(mpsb_ctx* ctx, const Gemm& g);
int set_boundary(mpsb_ctx* ctx, cd* p, cd v);
int op_orth_left(mpsb_ctx* ctx, cd* A, int Dl, int d, int Dr, cd* R /* Dr x Dr or null */);
int op_orth_right(mpsb_ctx* ctx, cd* A, int Dl, int d, int Dr);

// ---- sweeps (the reference's compress_* family)
int compress_var_apply_H_left(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain,
                              const mpsb_mps* A, const mpsb_mpo* H);
int compress_sum_var_apply_H(mpsb_ctx* ctx, bool right, mpsb_mps* A0, mpsb_env* const* env, mpsb_env* envop,
                             const mpsb_mps* Ain, const cd* coef, int numv, const mpsb_mps* const* A,
                             const mpsb_mpo* H);
int compress_sum_var_full(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const cd* coef, int numv,
                          const mpsb_mps* const* A, const mpsb_mpo* H /* null: compress_sum_var */, int maxsweeps);
int compress_var_apply_H(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain, const mpsb_mps* A,
                         const mpsb_mpo* H, int maxsweeps);
int ground_state_search(mpsb_ctx* ctx, mpsb_mps* At, const mpsb_mpo* H, int maxsweeps, double converge_rat,
                        double eigs_tol, double* ae);
int compression_svd(mpsb_ctx* ctx, const mpsb_mps* in, int dmax, double tol, std::vector<int64_t>& dims_out,
                    cd** sites, double* err_glob, double* err_trim, double* ent_ent);
int compress_two_site(mpsb_ctx* ctx, const mpsb_mps* Ain, const mpsb_mps* A, const mpsb_mpo* H, int maxsweeps,
                      double svd_tol, int dlim, std::vector<int64_t>& dims_out, std::vector<int64_t>& offs,
                      cd** sites);
int compress_two_site_sum(mpsb_ctx* ctx, const mpsb_mps* Ain, int numv, const cd* coef, const mpsb_mps* const* Av,
                          const mpsb_mpo* H, int maxsweeps, double svd_tol, int dlim, int mode,
                          std::vector<int64_t>& dims_out, std::vector<int64_t>& offs, cd** sites);
int rk4_step(mpsb_ctx* ctx, double dt, const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3,
             mpsb_mps* psi0, mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2, mpsb_mps* psi3, mpsb_env* env1,
             mpsb_env* env2, mpsb_env* env3, mpsb_env* envop);

}  // namespace mpsb
