/*
 * mpsb.h -- C ABI of the mpsb200 engine: the RK4 MPS/MPO time step of
 * jdnz/MatrixProductStates.jl on one B200 (sm_100a), complex128.
 *
 * Data conventions (the reference's own Julia layouts, so a Julia `ccall` can pass
 * `pointer(A[j])` directly):
 *   - complex numbers are interleaved (re, im) doubles  == Julia Complex{Float64}
 *   - every tensor is column-major:
 *       MPS site     A[chiL, d, chiR]                 (src/constructors.jl:19)
 *       MPO site     O[wL, d_out, wR, d_in]           (src/constructors.jl:239-243)
 *       3-index env  F[chi_A, w, chi_A0]              (src/constructors.jl:353)
 *       2-index env  F[chi_1, chi_2]                  (src/constructors.jl:369)
 *   - an MPS of `na` sites has bond dims dims[0..na] (dims[0] = dims[na] = 1);
 *     an MPO has channel dims w[0..na] (w[0] = w[na] = 1).
 *
 * Conventions of the interface:
 *   - every entry point returns int status: MPSB_OK (0) or a negative MPSB_ERR_*;
 *     mpsb_last_error() gives a message for the calling thread.
 *   - the library owns device memory behind opaque handles; the caller owns host buffers.
 *   - a context owns one CUDA stream; calls are asynchronous on it unless they return a
 *     host value (norms, scalar products), which synchronise.  A context is used by one
 *     host thread at a time.
 *   - there is no CPU fallback: without a usable sm_100 device, mpsb_ctx_create fails.
 */
#ifndef MPSB_H
#define MPSB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  MPSB_OK = 0,
  MPSB_ERR_INVALID_ARG = -1,      /* null handle / pointer, bad enum */
  MPSB_ERR_DIMENSION = -2,        /* shapes do not match (Julia: DimensionMismatch) */
  MPSB_ERR_CUDA = -3,             /* a CUDA runtime call failed */
  MPSB_ERR_OUT_OF_MEMORY = -4,    /* device allocation failed */
  MPSB_ERR_UNSUPPORTED = -5,      /* size outside what the kernels implement */
  MPSB_ERR_NONFINITE = -6,        /* a norm or probability came out NaN/Inf */
  MPSB_ERR_NO_DEVICE = -7         /* no CUDA device with compute capability 10.x */
};

typedef struct mpsb_ctx mpsb_ctx;
typedef struct mpsb_mps mpsb_mps;
typedef struct mpsb_mpo mpsb_mpo;
typedef struct mpsb_env mpsb_env;

/* ---------------------------------------------------------------- context */
const char* mpsb_last_error(void);
int mpsb_version(void);
int mpsb_ctx_create(int device, mpsb_ctx** out);
int mpsb_ctx_destroy(mpsb_ctx* ctx);
int mpsb_sync(mpsb_ctx* ctx);
/* Use an external CUDA stream (cudaStream_t passed as void*); NULL restores the own stream. */
int mpsb_ctx_set_stream(mpsb_ctx* ctx, void* stream);
/* Capture each RK4 step into a CUDA graph and replay it (default on). */
int mpsb_ctx_set_graphs(mpsb_ctx* ctx, int enable);
/* Overlap, inside mpsb_rk4stp_apply_H_half, each stage's environment initialisation with the
 * previous stage's sweep on a second stream (default on; MPSB_PIPELINE=0 in the environment
 * turns it off at context creation).  Results are identical either way; with it on, the
 * env1..env3 / envop buffers end up holding other stages' environments than the reference's
 * (they are scratch to every reference caller).  No reference counterpart. */
int mpsb_ctx_set_pipeline(mpsb_ctx* ctx, int enable);
/* Contraction precision of the sweep entry points (mpsb_rk4stp_apply_H_half, the
 * compress_* family).  slices = 0: FP64 (the default, the drop-in path).  slices = 3..7: each
 * complex GEMM of a sweep whose output spans at least `min_tiles` 128 x 32-complex tiles runs on
 * the int8 tensor pipe (tcgen05) with both operands written as `slices` 7-bit slices under a
 * per-row / per-column power-of-two scale, all slice products of equal weight accumulated
 * exactly in int32 and combined in FP64 (relative accuracy about 2^(-7 slices) of the
 * operands' row / column maxima); smaller GEMMs, the QR gauge moves, norms, MPO applies and
 * every observable stay FP64.  The reference computes in the element type of its arrays
 * (Complex{Float64}, or Complex{Float32} in its GPU examples,
 * examples/rydberg_density_matrix_gpu.jl:124-125); this setting has no direct counterpart. */
int mpsb_ctx_set_precision(mpsb_ctx* ctx, int slices, int min_tiles);
/* The sliced-path threshold of batched calls (calls on batch handles, no reference
 * counterpart): there a GEMM takes the int8 path when one copy's problem has at least
 * `min_flops` = 8 M N K real flops (and K >= 16), a rule that does not depend on the number of
 * copies, so a copy computes the same bits in a batch of any size.  Default 2^24.  The
 * autotuner of mpsb200.autotune picks it per bucket shape. */
int mpsb_ctx_set_batched_split_threshold(mpsb_ctx* ctx, double min_flops);
/* Device-time accounting of the sliced path's tensor-core GEMM kernel (no reference
 * counterpart): while enabled, every eager launch of that kernel is bracketed by CUDA events;
 * mpsb_ctx_profile_read waits for the context, returns the summed milliseconds, the number of
 * launches and their int8 operations since the last read, and clears them.  Launches inside
 * captured graphs are not counted. */
int mpsb_ctx_set_profiling(mpsb_ctx* ctx, int enable);
int mpsb_ctx_profile_read(mpsb_ctx* ctx, double* ms, int64_t* launches, double* int8_ops /* or NULL */);
/* Failure-detection self-test (no reference counterpart): one device thread waits `seconds`
 * (0 < seconds <= 10) on a barrier that nothing arrives on, with the bounded wait every pipeline
 * wait of this library uses; the wait runs out, the kernel sets the context's error word and
 * returns, and this call returns MPSB_ERR_CUDA with a "timed out" message.  The error word is
 * cleared by that report, and the context stays usable. */
int mpsb_wait_selftest(mpsb_ctx* ctx, double seconds);
/* Kernel launches issued by this context since creation (for accounting). */
int mpsb_ctx_launch_count(mpsb_ctx* ctx, int64_t* out);

/* ---------------------------------------------------------------- MPS (Vector{Array{T,3}}) */
int mpsb_mps_create(mpsb_ctx* ctx, int na, int d, const int64_t* dims /* na+1 */, mpsb_mps** out);
int mpsb_mps_destroy(mpsb_mps* A);
int mpsb_mps_info(const mpsb_mps* A, int* na, int* d, int64_t* dims /* na+1, may be NULL */);
/* site is 1-based like the reference; host buffer holds dims[site-1]*d*dims[site] complex.
 * set_site is ordered on the context stream and returns without waiting for it: a pageable
 * host buffer may be reused on return, a pinned one only after mpsb_sync.  get_site waits. */
int mpsb_mps_set_site(mpsb_mps* A, int site, const double* host);
int mpsb_mps_get_site(const mpsb_mps* A, int site, double* host);
/* device pointer of a site (for zero-copy interop); site 1-based */
int mpsb_mps_site_ptr(const mpsb_mps* A, int site, void** dptr);
/* dst .= copy.(src)  (examples/spin_model_quantum_trajectory_rk4.jl:130) */
int mpsb_mps_copy(mpsb_mps* dst, const mpsb_mps* src);

/* ---------------------------------------------------------------- batches of same-shape MPS
 * The batched trajectory engine (no reference counterpart: the reference runs one trajectory per
 * process, examples/spin_model_quantum_trajectory_rk4.jl:104-107).  A batch handle holds `batch`
 * copies of one MPS shape back to back; every entry point that takes MPS / environment handles
 * accepts batch handles of one common batch size (MPOs are shared by all copies) and runs each
 * kernel over all copies at once.  In calls on batch handles, or on views of one copy, every
 * per-kernel choice (a GEMM's split-K partition, the sliced path) depends on one copy's shape
 * only, so a copy computes the same bits in a batch of any size.  Copies are 0-based. */
int mpsb_mps_create_batch(mpsb_ctx* ctx, int na, int d, const int64_t* dims, int batch, mpsb_mps** out);
int mpsb_env_create_batch(mpsb_ctx* ctx, int na, const int64_t* dims1, const int64_t* dims2,
                          const int64_t* w /* na+1 or NULL */, int batch, mpsb_env** out);
int mpsb_mps_batch(const mpsb_mps* A, int* batch);
int mpsb_mps_set_site_copy(mpsb_mps* A, int copy, int site, const double* host);
int mpsb_mps_get_site_copy(const mpsb_mps* A, int copy, int site, double* host);
/* a handle on copy `copy` of a batch (shares its memory; destroy it before the batch) */
int mpsb_mps_view(mpsb_mps* A, int copy, mpsb_mps** out);
/* dst copy b <- srcs[which[b]] copy b (which[b] < 0 leaves copy b as it is): the per-trajectory
 * choice of A = copy(A_coh) / copy(A_r) / copy(A_l), examples/...rk4.jl:130-178 */
int mpsb_mps_select(mpsb_mps* dst, mpsb_mps* const* srcs, int nsrc, const int* which);
/* normalize_lo! of every copy; no[b] = its norm^2 before scaling */
int mpsb_normalize_lo_batch(mpsb_ctx* ctx, mpsb_mps* A, double* no);

/* ---------------------------------------------------------------- MPO (Vector{Array{T,4}}) */
int mpsb_mpo_create(mpsb_ctx* ctx, int na, int d, const int64_t* w /* na+1 */, mpsb_mpo** out);
int mpsb_mpo_destroy(mpsb_mpo* O);
/* same stream ordering as mpsb_mps_set_site */
int mpsb_mpo_set_site(mpsb_mpo* O, int site, const double* host);
int mpsb_mpo_get_site(const mpsb_mpo* O, int site, double* host);

/* ---------------------------------------------------------------- environments
 * build_env(TN, TA, dims1, dims2[, mpo_dims])  src/constructors.jl:347-375
 * w == NULL gives 2-index envs; ends are ones(1,1[,1]), interior zeros. */
int mpsb_env_create(mpsb_ctx* ctx, int na, const int64_t* dims1, const int64_t* dims2,
                    const int64_t* w /* na+1 or NULL */, mpsb_env** out);
int mpsb_env_destroy(mpsb_env* E);
/* entry is 1-based (1..na+1) like env[jj] in the reference */
int mpsb_env_get(const mpsb_env* E, int entry, double* host);
int mpsb_env_set(mpsb_env* E, int entry, const double* host);

/* ---------------------------------------------------------------- the RK4 hot path
 * RK4stp_apply_H_half!(dt, H, psi0, psi, psi1, psi2, psi3, env1, env2, env3, envop)
 *   src/timeevolution.jl:188-196 (11-arg); psi0 == psi gives the 10-arg in-place form
 *   src/timeevolution.jl:178-186.  H1, H2, H3 are H[1], H[2], H[3]. */
int mpsb_rk4stp_apply_H_half(mpsb_ctx* ctx, double dt,
                             const mpsb_mpo* H1, const mpsb_mpo* H2, const mpsb_mpo* H3,
                             mpsb_mps* psi0, mpsb_mps* psi, mpsb_mps* psi1, mpsb_mps* psi2,
                             mpsb_mps* psi3, mpsb_env* env1, mpsb_env* env2, mpsb_env* env3,
                             mpsb_env* envop);

/* compress_var_apply_H_left!(A0, envop, Ain, A, H)   src/compression.jl:321-347 */
int mpsb_compress_var_apply_H_left(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop,
                                   const mpsb_mps* Ain, const mpsb_mps* A, const mpsb_mpo* H);

/* compress_sum_var_apply_H_right!(A0, env, envop, Ain, coef, A, H)  src/compression.jl:1007-1063
 * compress_sum_var_apply_H_left!(A0, env, envop, Ain, coef, A, H)   src/compression.jl:889-944
 * numv = length(coef) = length(A); env has numv-1 entries; coef is numv interleaved complex;
 * A[numv-1] is the MPS the operator H acts on. A0 may equal A[0] (read before written). */
int mpsb_compress_sum_var_apply_H_right(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* const* env,
                                        mpsb_env* envop, const mpsb_mps* Ain, const double* coef,
                                        int numv, mpsb_mps* const* A, const mpsb_mpo* H);
int mpsb_compress_sum_var_apply_H_left(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* const* env,
                                       mpsb_env* envop, const mpsb_mps* Ain, const double* coef,
                                       int numv, mpsb_mps* const* A, const mpsb_mpo* H);

/* compress_var_apply_H!(A0, envop, Ain, A, H, maxsweeps)  src/compression.jl:217-258
 * (jump-operator application in the trajectory driver) */
int mpsb_compress_var_apply_H(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const mpsb_mps* Ain,
                              const mpsb_mps* A, const mpsb_mpo* H, int maxsweeps);

/* compress_sum_var_apply_H!(A0, envop, coef, A, H, maxsweeps)  src/compression.jl:805-887
 * maxsweeps R->L / L->R sweep pairs compressing sum_{l<numv-1} coef[l] A[l] + coef[numv-1] H A[numv-1]
 * into A0, which is both the initial guess and the output (it must not be one of the terms).
 * coef is numv interleaved complex; numv in 2..9.  The plain-term environments are internal. */
int mpsb_compress_sum_var_apply_H(mpsb_ctx* ctx, mpsb_mps* A0, mpsb_env* envop, const double* coef,
                                  int numv, mpsb_mps* const* A, const mpsb_mpo* H, int maxsweeps);

/* compress_sum_var(Ain, coef, A, maxsweeps)  src/compression.jl:496-565
 * The same without an operator (every term plain, numv in 1..8): A0 = the compression of
 * sum_l coef[l] A[l] with Ain as the initial guess (copied into A0 first unless A0 == Ain;
 * A0 must not be one of the terms).  The reference returns a new MPS; here the caller
 * passes the output handle. */
int mpsb_compress_sum_var(mpsb_ctx* ctx, mpsb_mps* A0, const mpsb_mps* Ain, const double* coef,
                          int numv, mpsb_mps* const* A, int maxsweeps);

/* ground_state_search!(At, H, maxsweeps, converge_rat, eigs_tol)  src/groundstate.jl:67-147
 * Single-site sweeps (left na..2, right 1..na-1, then site na) replacing each site by the
 * lowest eigenvector of its effective operator (A_prod_LOR_eigs, src/MatrixProductStates.jl:246-253)
 * and re-orthogonalising with the QR the reference uses; stops after a sweep whose last
 * eigenvalue has |ae| > converge_rat |ae at the sweep's first site| or |ae| < 1e-10.
 * The reference's ARPACK eigs(which=:SR) is replaced by Lanczos (full reorthogonalisation,
 * same tolerance rule); the eigenvector phase is fixed by <start|x> > 0.  *ae = last eigenvalue.
 * steady_state_search! (src/steadystate.jl:6-86) is this call with the product MPO Lconj*L. */
int mpsb_ground_state_search(mpsb_ctx* ctx, mpsb_mps* At, const mpsb_mpo* H, int maxsweeps,
                             double converge_rat, double eigs_tol, double* ae);

/* ---------------------------------------------------------------- gauge / norms
 * normalize_lo!(mps) src/orthonormalisation.jl:97-103 -> *no = sum(abs2, mps[end])
 * norm_lo(mps)       src/orthonormalisation.jl:117-121
 * leftorthonormalizationQR!(mps) src/orthonormalisation.jl:29-36 (returns the norm^2) */
int mpsb_normalize_lo(mpsb_ctx* ctx, mpsb_mps* A, double* no);
int mpsb_norm_lo(mpsb_ctx* ctx, const mpsb_mps* A, double* no);
int mpsb_leftorthonormalizationQR(mpsb_ctx* ctx, mpsb_mps* A, double* no);
/* leftorthogonalizeQR!(mps) src/orthonormalisation.jl:43-56: the same QR sweep with R carried
 * right, returning the norm^2 without rescaling (mpsproductstate / expandmps use this sweep) */
int mpsb_leftorthogonalizeQR(mpsb_ctx* ctx, mpsb_mps* A, double* no);
/* apply_site_operator!(A[site], op)  src/MatrixProductStates.jl:135-143; op is d x d column-major */
int mpsb_apply_site_operator(mpsb_ctx* ctx, mpsb_mps* A, int site, const double* op);

/* ---------------------------------------------------------------- observables
 * scal_prod(A, B)          src/MatrixProductStates.jl:345-358   <A|B>
 * scal_op_prod(A, O, B)    src/MatrixProductStates.jl:327-340   <A|O|B>
 * scal_prod_no_conj(A, B)  src/MatrixProductStates.jl:366-379   sum A.B (no conjugation)
 * measure_local(A, op)     examples/spin_model_quantum_trajectory_rk4.jl:220-231
 *                          (measure_excitations!: right-to-left local_exp sweep, mps_base.jl:341-349),
 *                          out[na] = real(local <op_n>) for a left-orthonormal MPS. */
int mpsb_scal_prod(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mps* B, double* out /* 2 */);
int mpsb_scal_op_prod(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mpo* O, const mpsb_mps* B,
                      double* out /* 2 */);
int mpsb_scal_prod_no_conj(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mps* B, double* out /* 2 */);
int mpsb_measure_local(mpsb_ctx* ctx, const mpsb_mps* A, const double* op /* d x d */, double* out);

/* applyMPOtoMPS(mps, mpo)  src/MatrixProductStates.jl:115-133 (exact, bond dims multiply);
 * out must have dims[k]*w[k] bonds. */
int mpsb_apply_mpo_to_mps(mpsb_ctx* ctx, const mpsb_mps* A, const mpsb_mpo* O, mpsb_mps* out);

/* ---------------------------------------------------------------- op level (device pointers)
 * Raw device buffers in the Julia layouts above, for op-by-op parity checks and for callers
 * that manage their own memory.  Outputs are written, never accumulated. */
/* prod_AOR(A, O, R) -> AOR[chiL, wL, d, chiR0]      src/mps_base.jl:7-19 */
int mpsb_op_prod_AOR(mpsb_ctx* ctx, const void* A, const void* O, const void* R, void* AOR,
                     int chiL, int d, int chiR, int wL, int wR, int chiR0);
/* prod_AOL(A, O, L) -> AOL[chiL0, d, chiR, wR]      src/mps_base.jl:26-39 */
int mpsb_op_prod_AOL(mpsb_ctx* ctx, const void* A, const void* O, const void* L, void* AOL,
                     int chiL, int d, int chiR, int wL, int wR, int chiL0);
/* prod_LR!(A0, L, AOR): A0[chiL0, d, chiR0] = L' * AOR   src/mps_base.jl:53-61 */
int mpsb_op_prod_LR_3_4(mpsb_ctx* ctx, const void* L, const void* AOR, void* A0,
                        int chiL, int wL, int chiL0, int d, int chiR0);
/* prod_LR!(A0, AOL, R): A0 = AOL * R                     src/mps_base.jl:73-81 */
int mpsb_op_prod_LR_4_3(mpsb_ctx* ctx, const void* AOL, const void* R, void* A0,
                        int chiL0, int d, int chiR, int wR, int chiR0);
/* update_re!(env, A0, AOR): env[chiL, wL, chiL0]         src/mps_base.jl:151-160 */
int mpsb_op_update_re(mpsb_ctx* ctx, const void* A0, const void* AOR, void* env,
                      int chiL, int wL, int d, int chiR0, int chiL0);
/* update_le!(env, A0, AOL): env[chiR, wR, chiR0]         src/mps_base.jl:232-241 */
int mpsb_op_update_le(mpsb_ctx* ctx, const void* A0, const void* AOL, void* env,
                      int chiL0, int d, int chiR, int wR, int chiR0);
/* prod_AOR for callers that cannot allocate device memory. No counterpart in the reference:
 * it exists for hosts whose device memory belongs to their own pool allocator (a Julia
 * CUDA.jl or PyTorch caching allocator) or that must not call cudaMalloc/cudaFree in their
 * time loop, since those synchronise the device.  Same result as mpsb_op_prod_AOR, but it
 * takes a CUDA stream (cudaStream_t as void*) instead of a context and calls no cudaMalloc,
 * cudaFree or allocating routine: its one intermediate, A*R, lives in a fixed 16 MiB array
 * compiled into the library (held on every GPU that loads the library until exit), so
 * chiL*d*wR*chiR0 must be <= 1048576, else it returns MPSB_ERR_UNSUPPORTED.  The first call
 * on a device looks up that array's device address (make the device current first, and make
 * that first call before any stream capture).  All calls share the array: calls that overlap
 * on the GPU (other streams, other host threads) race; serialise them on one stream. */
int mpsb_op_prod_AOR_noalloc(void* stream, const void* A, const void* O, const void* R, void* AOR,
                             int chiL, int d, int chiR, int wL, int wR, int chiR0);
/* compressionSVD!(mps, dmax, tol)  src/compression.jl:1280-1312 -- the truncation rule
 * chi_new = min(#{cumsum(s^2/sum s^2) < 1 - tol} + 1, dmax) applied site by site from the right
 * to a left-canonical MPS.  The reference resizes mps in place; here the result (right
 * canonical, new bond dims) is a new handle *out.  err_trim and ent_ent (na values, host) and
 * *err_glob are the reference's return values. */
int mpsb_compression_svd(mpsb_ctx* ctx, const mpsb_mps* in, int dmax, double tol, mpsb_mps** out,
                         double* err_glob, double* err_trim, double* ent_ent);

/* compress_var_apply_H_two_site(Ain, A, H, maxsweeps, svd_tol, dims, dlim)  src/compression.jl:355-411
 * Two-site variational compression of H*A (guess Ain, left canonical) with a thin SVD of each
 * pair tensor truncated by the compressionSVD! rule; the bond dims adapt (<= dlim), so the
 * result is a new handle *out (its dims are the reference's updated `dims`).  The reference's
 * version calls the undefined `svdecon` and contracts its stored-conjugated left environment
 * unconjugated; this one uses the thin SVD and the single-site path's conjugation.
 * compress_var_two_site (src/compression.jl:110-165) is this call with an identity MPO. */
int mpsb_compress_var_apply_H_two_site(mpsb_ctx* ctx, const mpsb_mps* Ain, const mpsb_mps* A,
                                       const mpsb_mpo* H, int maxsweeps, double svd_tol, int dlim,
                                       mpsb_mps** out);

/* compress_sum_var_apply_H_two_site(Ain, coef, A, H, maxsweeps, svd_tol, dims, dlim)
 *   src/compression.jl:1072-1157 (half = 0), its _left form :1159-1215 (half = 1: one R->L
 *   sweep, first site U diag(S)) and _right form :1218-1276 (half = 2: one L->R sweep from the
 *   right environments of a right-canonical Ain, coefficients on the left boundary; the
 *   operator term's is stored conjugated there, since that environment is contracted
 *   conjugated, so the result is the stated sum also for complex coefficients);
 * compress_sum_var_two_site(Ain, coef, A, maxsweeps, svd_tol, dims, dlim)  :574-648 when H is NULL.
 * Two-site variational compression of sum_l coef[l] A[l], the last term through H when H is
 * given; coef is numv interleaved complex (at most 8 plain terms besides the H term); the terms
 * may have different bond dims; Ain is the left-canonical guess (right-canonical for
 * half = 2).  Bond dims adapt (<= dlim): the result is a new handle *out.  As in
 * mpsb_compress_var_apply_H_two_site the undefined `svdecon` is the thin SVD and the pair
 * contractions use the environments as the single-site path does (the reference's
 * A_prod_LR_two_site, src/MatrixProductStates.jl:288-292, contracts the stored left
 * environment on its A0 index, i.e. transposed). */
int mpsb_compress_sum_var_apply_H_two_site(mpsb_ctx* ctx, const mpsb_mps* Ain, const double* coef, int numv,
                                           const mpsb_mps* const* A, const mpsb_mpo* H, int maxsweeps,
                                           double svd_tol, int dlim, int half, mpsb_mps** out);

/* svd(M) as compressionSVD! calls it (src/compression.jl:1296): thin SVD X = U diag(S) V^H of a
 * device m x n column-major matrix, k = min(m, n); U (m x k) and V (n x k) device, S (k) host,
 * singular values descending.  One-sided Jacobi (relative accuracy); phases of the singular
 * vectors are those of the rotation sequence (LAPACK's are equally arbitrary). */
int mpsb_op_svd(mpsb_ctx* ctx, const void* X, void* U, double* S, void* V, int m, int n);

/* Q of the LAPACK geqrf+orgqr QR of the column-major m x n matrix X (m >= n):
 * qrq!(X)  src/orthonormalisation.jl:180-184. Q may alias X. R (n x n) optional (NULL). */
int mpsb_op_qr(mpsb_ctx* ctx, const void* X, void* Q, void* R, int m, int n);
/* C = alpha op(A) op(B) + beta C on device buffers with element strides (complex128;
 * op = conjugate when conjA / conjB), the GEMM every contraction of src/mps_base.jl reduces to
 * (BLAS zgemm there).  slices = 0: FP64 (DMMA); 3..7: the int8-sliced tensor-core path of
 * mpsb_ctx_set_precision.  alpha / beta: interleaved complex, NULL = 1 / 0. */
int mpsb_op_zgemm(mpsb_ctx* ctx, int M, int N, int K, const void* A, int64_t a_m, int64_t a_k, int conjA,
                  const void* B, int64_t b_k, int64_t b_n, int conjB, void* C, int64_t c_m, int64_t c_n,
                  const double* alpha, const double* beta, int slices);

#ifdef __cplusplus
}
#endif
#endif /* MPSB_H */
