/*
 * imps_b200 -- C ABI of the B200 implementation of the InfiniteMPSAlgorithms
 * VUMPS / IDMRG / TDVP inner loop (guochu/InfiniteMPSAlgorithms).
 *
 * Every entry point takes plain pointers and sizes.  Tensors are column-major
 * ComplexF64 arrays (interleaved re, im doubles), i.e. exactly the memory of a
 * Julia `Array{ComplexF64}` of the reference, so a Julia `ccall` passes
 * `pointer(A)` directly.  Device memory is owned by the library behind the
 * opaque handles below; `*_dev` entry points take device pointers instead.
 *
 * Index conventions (reference src/algorithms/groundstates/effective.jl:3-5):
 *   site tensors A[a, s, b]       shape (Dl, d, Dr)
 *   left envs    GL[bra, w, ket]  shape (Dl, m, Dl)
 *   right envs   GR[ket, w, bra]  shape (Dr, n, Dr)
 *   MPO tensors  W[wl, u, wr, s]  shape (m, d, n, d), u = output (bra) leg
 *
 * Return value: an IMPS_* status.  IMPS_NOT_CONVERGED is a warning (the
 * reference only emits `@warn`), the result is still written.
 *
 * Threading: a context owns one CUDA stream; calls on one context must be
 * serialised by the caller (one context per host thread).
 */
#ifndef IMPS_B200_H
#define IMPS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  IMPS_OK = 0,
  IMPS_NOT_CONVERGED = 1,   /* warning: iteration limit reached, result written   */
  IMPS_DIM_MISMATCH = -1,   /* reference: DimensionMismatch                        */
  IMPS_INVALID_ARG = -2,    /* reference: ArgumentError                            */
  IMPS_OOM = -3,            /* device allocation failed                            */
  IMPS_CUDA_ERROR = -4,     /* CUDA / cuSOLVER failure                             */
  IMPS_TIMEOUT = -5,        /* a bounded device wait gave up                       */
  IMPS_NO_DEVICE = -6       /* no CUDA device visible                              */
};

/* Precision modes of the Heff / transfer contractions. */
enum {
  IMPS_PREC_FP64 = 0,       /* plain method: FP64 end to end                       */
  IMPS_PREC_SPLIT_I8 = 1    /* int8 split products on tcgen05, exact int32 sums    */
};

/* Field selectors for imps_state_get / imps_state_set. */
enum { IMPS_AL = 0, IMPS_AR = 1, IMPS_C = 2, IMPS_AC = 3 };

typedef struct imps_ctx imps_ctx;
typedef struct imps_mpo imps_mpo;
typedef struct imps_state imps_state;
typedef struct imps_envs imps_envs;
typedef struct imps_mult_envs imps_mult_envs;

/* KrylovKit `ConvergenceInfo` equivalent (converged, numiter, numops, normres). */
typedef struct {
  int32_t converged;
  int32_t numiter;
  int32_t numops;
  int32_t pad;
  double normres;
  double value_re;   /* eigenvalue (eigsolve) */
  double value_im;
} imps_krylov_info;

/* Per-build statistics of the environment solver. */
typedef struct {
  int32_t solves;
  int32_t gmres_iters;
  int32_t gmres_ops;
  int32_t pushes;
  int32_t converged;   /* 1 when every linsolve met its tolerance */
  int32_t pad;
  double max_normres;
} imps_env_info;

/* Gauge-fixing iteration summary (uniform_leftorth!/uniform_rightorth!). */
typedef struct {
  int32_t niter;
  int32_t converged;
  double err;
} imps_gauge_info;

/* One VUMPS iteration summary. */
typedef struct {
  double galerkin;            /* calc_galerkin after the iteration              */
  double energy_re;           /* expectationvalue(psi, H, envs)                 */
  double energy_im;
  int32_t ac_matvecs;         /* AC Heff applications in the eigensolves        */
  int32_t c_matvecs;
  int32_t gauge_iters;
  int32_t env_gmres_ops;
  imps_env_info env;
} imps_vumps_info;

/* ---------------------------------------------------------------- context */
/* Replaces: the implicit Julia process state (no reference counterpart). */
int imps_ctx_create(int device, imps_ctx** out);
int imps_ctx_destroy(imps_ctx* ctx);
/* Use a caller-owned cudaStream_t (e.g. the host framework's current stream). */
int imps_ctx_set_stream(imps_ctx* ctx, void* cuda_stream);
/* Precision of the Heff/transfer contractions: IMPS_PREC_FP64 or
 * IMPS_PREC_SPLIT_I8 with `nslices` int8 slices per operand (2..8, each slice adding
 * 7 bits); nslices <= 0 selects slices per call from the requested solver tolerance
 * (up to 6; a tolerance that needs more runs the FP64 engine). */
int imps_ctx_set_precision(imps_ctx* ctx, int mode, int nslices);
int imps_ctx_synchronize(imps_ctx* ctx);
/* Bound of each pipeline wait inside the split GEMM kernel, in SM clock cycles
 * (0 restores the default 2e9, about 1 s).  A wait that runs out sets a device
 * error flag and the kernel returns early; the flag is read at the context's next
 * host synchronisation (at the latest when the entry point returns) and the call
 * returns IMPS_TIMEOUT; the context stays usable.  No reference counterpart (the
 * reference has no device code): the bounded-wait failure detection of this
 * library. */
int imps_ctx_set_wait_limit(imps_ctx* ctx, int64_t cycles);
/* Cap (bytes, 0 = none) on the context's scratch workspace: the grow-only device
 * buffers the solvers and contractions keep between calls (Krylov bases, Heff
 * intermediates, gauge work arrays).  A call that would grow it past the cap
 * returns IMPS_OOM and leaves the context usable; imps_ctx_workspace_bytes reports
 * the current size.  Object storage (states, environments, MPOs) and the cached
 * int8 operand splits are not counted.  No reference counterpart (Julia's GC owns
 * the reference's arrays). */
int imps_ctx_set_workspace_limit(imps_ctx* ctx, int64_t bytes);
int imps_ctx_workspace_bytes(imps_ctx* ctx, int64_t* bytes);
const char* imps_ctx_last_error(const imps_ctx* ctx);
const char* imps_status_string(int status);
/* Kernel timing with CUDA events on the context stream, per kernel class. */
int imps_ctx_profile(imps_ctx* ctx, int enable);
int imps_ctx_profile_get(imps_ctx* ctx, const char* kernel_class, int64_t* launches, double* total_ms,
                         double* work);
int imps_ctx_profile_reset(imps_ctx* ctx);
/* Restrict timing to a comma-separated list of kernel classes (NULL or "" = all). */
int imps_ctx_profile_classes(imps_ctx* ctx, const char* csv);
/* Every kernel class seen so far as text lines "class[@call-site] launches total_ms work". */
int imps_ctx_profile_dump(imps_ctx* ctx, char* buf, int64_t len);
/* counters[0..7] (8 entries) = AC applies, C applies, pushes, GEMM launches, all kernel launches,
 * QRpos/LQpos factorizations, real flops of all complex GEMMs (8 M N K each), real flops of
 * the QR factorizations */
int imps_ctx_counters(imps_ctx* ctx, int64_t* counters);
/* The same counters followed by [8] split GEMM launches, [9] their algorithmic real
 * flops (8 M N K of each complex product) and [10] the int8 operations the tensor
 * pipe executed for them; n entries are written (entries past 10 read 0). */
int imps_ctx_counters_ext(imps_ctx* ctx, int64_t* counters, int n);

/* -------------------------------------------------------------------- MPO */
/* Replaces SparseIMPO / SchurMPOTensor storage (src/operators/mpohamiltonian.jl:33-52):
 * W[l] is the dense tompotensor(H[l]) of shape (m[l], d[l], n[l], d[l])
 * (src/algorithms/groundstates/envs.jl:332). */
int imps_mpo_create(imps_ctx* ctx, int N, const int* m, const int* d, const int* n, const double* const* W,
                    imps_mpo** out);
int imps_mpo_destroy(imps_mpo* mpo);

/* ------------------------------------------------------------------ state */
/* Replaces CanonicalIMPS (src/states/canonicalmps.jl:17-40).  chi[l] is the
 * bond dimension right of site l (bond N-1 == bond 0), d[l] the physical dim. */
int imps_state_create(imps_ctx* ctx, int N, const int* d, const int* chi, imps_state** out);
int imps_state_destroy(imps_state* st);
int imps_state_set(imps_state* st, int field, int site, const double* host);
int imps_state_get(const imps_state* st, int field, int site, double* host);
int imps_state_copy(imps_state* dst, const imps_state* src);
/* CanonicalIMPS(As): gaugefix!(:LR) from C0 = I, AC = AL*C
 * (src/states/canonicalmps.jl:151-170). */
int imps_state_canonicalize(imps_state* st, const double* const* As, double tol, int maxiter,
                            imps_gauge_info* info);
/* CanonicalIMPS(ALs, C0): gaugefix!(:R), AC = AL*C (src/states/canonicalmps.jl:180-195). */
int imps_state_from_al(imps_state* st, const double* const* ALs, const double* C0, double tol, int maxiter,
                       imps_gauge_info* info);
/* gauge_step! (src/algorithms/groundstates/vumps.jl:23-31): keep st->AL, right gauge
 * fix from C0 = st->C[N] for AR and C, then AC = AL*C. */
int imps_gauge_step(imps_state* st, double tol, int maxiter, imps_gauge_info* info);
/* dot(psi, psi) (src/states/canonicalmps.jl:262-269). */
int imps_state_dot(imps_state* st, double* re, double* im);

/* ------------------------------------------------------------ environments */
/* Replaces DMRGCache(psi, ::SparseIMPO) (src/algorithms/groundstates/envs.jl:248-257, 321-518). */
int imps_envs_create(imps_ctx* ctx, const imps_state* st, const imps_mpo* mpo, imps_envs** out);
int imps_envs_destroy(imps_envs* envs);
/* DMRGCache constructor / recalculate! (envs.jl:321-546); warm != 0 uses the
 * current contents as init_lefts / init_rights. */
int imps_envs_build(imps_envs* envs, const imps_state* st, const imps_mpo* mpo, double tol, int maxiter,
                    int krylovdim, int warm, imps_env_info* info);
/* side 0: lefts[site], side 1: rights[site] */
int imps_envs_get(const imps_envs* envs, int side, int site, double* host);
int imps_envs_set(imps_envs* envs, int side, int site, const double* host);

/* ------------------------------------------------- effective Hamiltonians */
/* MPO_AC_Hamiltonian action (src/algorithms/groundstates/effective.jl:66-68, 90-102). */
int imps_ac_apply(imps_envs* envs, const imps_mpo* mpo, int site, const double* x, double* y);
int imps_ac_apply_dev(imps_envs* envs, const imps_mpo* mpo, int site, const void* x_dev, void* y_dev);
/* Allocation-free AC apply -- no counterpart in the reference.  For callers that
 * cannot let the library call cudaMalloc (their caching allocator already holds
 * the device memory, or they must avoid the implicit synchronisation of
 * cudaMalloc/cudaFree): the same FP64 GL.x -> level mix -> .GR pipeline as
 * imps_ac_apply, every intermediate held in one fixed 64 MiB device array of the
 * library (per device, kept until exit).  GL (Dl, m, Dl), GR (Dr, n, Dr), x, y
 * (Dl, d, Dr) are caller-owned device buffers, W_host the (m, d, n, d) MPO tensor
 * in host memory (<= 64 KiB).  Sizes needing more than the array
 * (16*Dl*d*Dr*(m+n) bytes) return IMPS_INVALID_ARG.  All calls share the array:
 * calls whose GPU work overlaps race.  The array is created (and its address
 * looked up) by imps_ctx_create on the context's device, so create the context
 * before the caller's allocator reserves the device memory.  The call is
 * asynchronous: the work is queued on the context's stream and the call returns
 * before it finishes; order GL, GR, x and y against that stream (or pass the
 * caller's stream to imps_ctx_set_stream).  W_host is copied during the call. */
int imps_ac_apply_noalloc(imps_ctx* ctx, int Dl, int d, int Dr, int m, int n, const double* W_host,
                          const void* GL_dev, const void* GR_dev, const void* x_dev, void* y_dev);
/* MPO_C_Hamiltonian action (effective.jl:52-54, 72-76): GL = lefts[site+1], GR = rights[site]. */
int imps_c_apply(imps_envs* envs, int site, const double* x, double* y);
int imps_c_apply_dev(imps_envs* envs, int site, const void* x_dev, void* y_dev);

/* --------------------------------------------------------- transfer pushes */
/* push_env_left(L, above, below) / push_env_right(R, above, below)
 * (src/transfermatrix.jl:5-7, 23-26, 54-66); above, below: (Dl, d, Dr). */
int imps_push_left(imps_ctx* ctx, int Dl, int d, int Dr, const double* L, const double* above,
                   const double* below, double* out);
int imps_push_right(imps_ctx* ctx, int Dl, int d, int Dr, const double* R, const double* above,
                    const double* below, double* out);
/* Schur MPO pushes (envs.jl:199-231, transfer_leftenv!/transfer_rightenv! :591-604)
 * with the MPO tensor of site `site`. */
int imps_push_mpo_left(imps_ctx* ctx, const imps_mpo* mpo, int site, int Dl, int Dr, const double* L,
                       const double* A, double* out);
int imps_push_mpo_right(imps_ctx* ctx, const imps_mpo* mpo, int site, int Dl, int Dr, const double* R,
                        const double* A, double* out);

/* ------------------------------------------------------------------- GEMM */
/* C = alpha op(A) op(B) + beta C on device pointers (column-major complex128),
 * op: 0 = N, 1 = T, 2 = C (conjugate transpose), through the context's precision
 * engine: the @tensor contractions of the reference (TensorOperations -> BLAS
 * ZGEMM, src/InfiniteMPSAlgorithms.jl:260) run here. */
int imps_zgemm(imps_ctx* ctx, int opA, int opB, int M, int N, int K, double alpha_re, double alpha_im,
               const void* A, int64_t lda, const void* B, int64_t ldb, double beta_re, double beta_im, void* C,
               int64_t ldc);

/* --------------------------------------------------------- factorizations */
/* leftorth(M; alg = QRpos()) / rightorth(M; alg = LQpos()) (FiniteMPSAlgorithms,
 * used at src/states/ortho.jl:150, 188, 214-225).  M is m x n column-major. */
int imps_qrpos(imps_ctx* ctx, int m, int n, const double* M, double* Q, double* R);
int imps_lqpos(imps_ctx* ctx, int m, int n, const double* M, double* L, double* Q);
/* regauge!(AC, C) (src/states/ortho.jl:214-219): AL = Q(AC) Q(C)^H. */
int imps_regauge(imps_ctx* ctx, int Dl, int d, int Dr, const double* AC, const double* C, double* AL);

/* ----------------------------------------------------------- Krylov solvers */
/* fixedpoint(H_AC, x0, :SR, Lanczos) (src/utility.jl:180-186, 379-393). */
int imps_eigsolve_ac(imps_envs* envs, const imps_mpo* mpo, int site, const double* x0, double* x, double tol,
                     int krylovdim, int maxiter, int eager, imps_krylov_info* info);
int imps_eigsolve_c(imps_envs* envs, int site, const double* x0, double* x, double tol, int krylovdim,
                    int maxiter, int eager, imps_krylov_info* info);
/* integrate(H, x, dt, Lanczos) -> exponentiate (src/algorithms/timeevo/tdvp.jl:14-20). */
int imps_exponentiate_ac(imps_envs* envs, const imps_mpo* mpo, int site, double dt_re, double dt_im,
                         const double* x0, double* x, double tol, int krylovdim, int maxiter,
                         imps_krylov_info* info);
int imps_exponentiate_c(imps_envs* envs, int site, double dt_re, double dt_im, const double* x0, double* x,
                        double tol, int krylovdim, int maxiter, imps_krylov_info* info);
/* linsolve / integrate on a diagonal operator diag(dvals) of length n (the
 * reference's solver-level known-answer tests, test/algorithms/api.jl:248-251, 469-478). */
int imps_linsolve_diag(imps_ctx* ctx, int64_t n, const double* dvals, const double* b, const double* x0,
                       double a0, double a1, double tol, int krylovdim, int maxiter, double* x,
                       imps_krylov_info* info);
int imps_exponentiate_diag(imps_ctx* ctx, int64_t n, const double* dvals, double dt_re, double dt_im,
                           const double* x0, double* x, double tol, int krylovdim, int maxiter,
                           imps_krylov_info* info);

/* ------------------------------------------------------------- observables */
/* calc_galerkin (src/algorithms/groundstates/vumps.jl:111-124). */
int imps_galerkin(imps_envs* envs, const imps_mpo* mpo, const imps_state* st, double* eps);
/* expectationvalue(psi, H::SparseIMPO, envs) (src/observables/expval.jl:93-112). */
int imps_energy(imps_envs* envs, const imps_mpo* mpo, imps_state* st, double* re, double* im);
/* expectationvalue(psi, (site,) => O) (src/observables/expval.jl:33-37); O is d x d. */
int imps_local_expval(imps_state* st, int site, const double* O, double* re, double* im);

/* ------------------------------------- dense-MPO channel and observables */
/* dominant_env([W,] psi; side) (src/algorithms/groundstates/envs.jl:34-99): dominant
 * (:LM) eigenvector of the transfer matrix of one unit cell, identity channel (AL / AR
 * pushes) when mpo is NULL, else the dense-MPO channel of `mpo` (the tompotensors taken
 * as a DenseIMPO); side 0 = left, 1 = right.  Arnoldi from v0 = ones; L_host receives
 * the unit-norm (D, w, D) environment (w = 1 for the identity channel), lambda[0..1]
 * the eigenvalue. */
int imps_dominant_env(imps_state* st, const imps_mpo* mpo, int side, double tol, int krylovdim, int maxiter,
                      double* lambda, double* L_host, imps_krylov_info* info);
/* DMRGCache(psi, ::DenseIMPO) (envs.jl:284-304): dominant left / right environments
 * pushed around the unit cell, then normalize_envs! (envs.jl:559-584). */
int imps_envs_build_dense(imps_envs* envs, imps_state* st, const imps_mpo* mpo, double tol, int krylovdim,
                          int maxiter, imps_krylov_info* info);
/* expectationvalue(psi, ::DenseIMPO, envs) (src/observables/expval.jl:60-79). */
int imps_energy_dense(imps_envs* envs, const imps_mpo* mpo, imps_state* st, double* re, double* im);
/* correlator(psi, O1, O2, i, js) (src/observables/correlators.jl:13-42): <O1_i O2_j> /
 * <psi|psi> for the nj increasing 1-based sites js (> i); O1, O2 are d x d column-major
 * complex; out receives nj interleaved complex values.  As in the reference, a later j
 * transfers through AR from the previous j + 1 on. */
int imps_correlator(imps_state* st, const double* O1, const double* O2, int i, int nj, const int* js, double* out);
/* Truncated thin SVD M = U diag(s) V^H of the host matrix M (m x n, column-major complex)
 * by one-sided Jacobi on the device (the tsvd of the two-site splits; FiniteMPSAlgorithms
 * `tsvd`, used at src/algorithms/groundstates/idmrg.jl:107-111): s descending, at most
 * kmax (> 0, else min(m, n)) values kept and those above `cutoff` (at least one); U
 * (m x k), s (k), V (n x k) caller-owned with room for min(m, n) columns; *k receives k. */
int imps_svd(imps_ctx* ctx, int m, int n, const double* M, int kmax, double cutoff, double* U, double* s, double* V,
             int* k);
/* entanglement_spectrum(psi, loc) (src/observables/toolbox.jl:9-14) of bond `bond`
 * (0-based, bond l right of site l): the chi normalised squared singular values of C,
 * descending (one-sided Jacobi on the device); p holds chi doubles. */
int imps_entanglement_spectrum(imps_state* st, int bond, double* p);

/* timeevompo(H::SparseIMPO, delta, WI()/WII()) (src/algorithms/timeevo/w1w2.jl:26-45),
 * one site: from the Schur tensor W (m, d, n, d) (level 1 and level m = n the identity
 * levels) the W^I (alg = 1) or W^II (alg = 2) tensor (m-1, d, n-1, d) of the dense
 * MPO approximating exp(delta H), by the block-exponential construction of
 * arXiv:1407.1832 (the reference's own kernel is in an unvendored package).  Host
 * computation, needs no device; out is caller-owned. */
int imps_timeevompo_tensor(int m, int d, int n, const double* W, double delta_re, double delta_im, int alg,
                           double* out);

/* ---------------------------------------------------------------- gradients */
/* No counterpart in the reference (an extension for gradient-based iMPS
 * optimisation).  Both use the environments in `envs`, which must be the fixed
 * points for `st` and `mpo` (after imps_envs_build); the right environments are
 * the solution of the adjoint of the left fixed-point system, so neither call
 * iterates.  The state is taken as normalised (every canonical state is).
 * G (host, interleaved complex, column-major (m, d, n, d)) = dE/dW[site]: the
 * derivative of imps_energy's E with respect to each entry of the site's dense
 * MPO tensor; the two identity blocks of the Schur form (level 1 -> 1 and
 * m -> n) are returned as zero.  dE/dtheta for a coupling theta is
 * sum(dW/dtheta * G) over the sites. */
int imps_energy_grad_mpo(imps_envs* envs, const imps_mpo* mpo, imps_state* st, int site, double* G);
/* g (host, interleaved complex, (Dl, d, Dr)) = dE/dconj(AL[site]) of the normalised
 * energy of the uniform MPS generated by AL: (H_AC(AC) - lambda AC) C[site]^H with
 * lambda = <AC|H_AC|AC>/<AC|AC>.  A real direction X changes E by 2 Re <g, X>. */
int imps_energy_grad_al(imps_envs* envs, const imps_mpo* mpo, imps_state* st, int site, double* g);

/* -------------------------------------------------------------- algorithms */
/* localupdate_step! (vumps.jl:7-19): per site AC and C eigensolves + regauge!,
 * candidate ALs written into st->AL. */
int imps_vumps_localupdate(imps_envs* envs, const imps_mpo* mpo, imps_state* st, double tol, int krylovdim,
                           int maxiter, int eager, int32_t* ac_matvecs, int32_t* c_matvecs);
/* One full VUMPS iteration (vumps.jl:51-85) for the outer-loop index `iter`
 * (1-based) and the previous Galerkin error `eps`, with the reference's dynamic
 * tolerances (Defaults, src/utility.jl:308-320). */
/* Batched group of imps_vumps_iter calls over n independent instances (e.g. many
 * Hamiltonians with uneven bond dimensions).  Instances on distinct contexts run
 * concurrently, one host thread and one stream per context (at most nthreads
 * threads; <= 0 means 16); instances sharing a context run in order.  status[i] is
 * each instance's own status; the return value is the most severe error, else
 * IMPS_OK.  No counterpart in the reference, whose instances would be separate
 * find_groundstate calls (vumps.jl:51-85). */
int imps_vumps_iter_batch(int n, imps_envs* const* envs, const imps_mpo* const* mpos, imps_state* const* states,
                          const int* iters, const double* eps, imps_vumps_info* infos, int* status, int nthreads);
int imps_vumps_iter(imps_envs* envs, const imps_mpo* mpo, imps_state* st, int iter, double eps,
                    imps_vumps_info* info);
/* timestep(psi, H, dt, TDVP(), envs) (src/algorithms/timeevo/tdvp.jl:34-53). */
int imps_tdvp_step(imps_envs* envs, const imps_mpo* mpo, imps_state* st, double dt_re, double dt_im,
                   double tol, int krylovdim, int maxiter, double gauge_tol, int gauge_maxiter,
                   imps_krylov_info* info);
/* _localupdate_sweep_idmrg! (src/algorithms/groundstates/idmrg.jl:12-33); returns the
 * last eigenvalue in *E and ||C[0] - C_old|| in *eps. */
int imps_idmrg_sweep(imps_envs* envs, const imps_mpo* mpo, imps_state* st, double tol, int krylovdim,
                     int maxiter, int eager, double* E, double* eps);
/* _localupdate_sweep_idmrg2! (src/algorithms/groundstates/idmrg.jl:113-185) with
 * trunc = truncdim(D) (_idmrg2_split, idmrg.jl:107-111): two-site windows L->R as :ACAR,
 * the wrap window as :ALAC, R->L as :ALAC, the closing window as :ACAR.  Bond dimensions
 * change in place (k = min(D, Dl d1, d2 Dr) at every split; read them back with
 * imps_state_bonds).  Requires N >= 2 (ArgumentError otherwise).  *E = eigenvalue of the
 * closing window, *eps = ||C[0] - C_old|| (diagonals zero-padded when their sizes differ;
 * the reference's norm of a difference assumes equal sizes).  FP64 throughout. */
int imps_idmrg2_sweep(imps_envs* envs, const imps_mpo* mpo, imps_state* st, int D, double tol, int krylovdim,
                      int maxiter, int eager, double* E, double* eps);
/* y = AC2_hamiltonian(p) * x for the window (p, p+1), 0-based p, x and y (Dl, d1, d2, Dr)
 * column-major on the host (MPO_AC2_Hamiltonian action, effective.jl:160-197). */
int imps_ac2_apply(imps_envs* envs, const imps_mpo* mpo, int p, const double* x, double* y);
/* chi[l] = bond dimension right of site l, l = 0..N-1 (bonddim(psi, l+1)). */
int imps_state_bonds(const imps_state* st, int* chi);

/* ---- MPO application mult(W, psi, VOMPS(D)) (src/algorithms/arithmetics/mult.jl) ----
 * W is any imps_mpo used as a dense MPO (the DenseIMPO channel: AL = AR = AC = W, C = I).
 *
 * svdguess_mult(W, psi, D) then CanonicalIMPS(...) (mult.jl:848-870, compress.jl:161-190):
 * the product's site tensors streamed right to left from psi.AL with every bond truncated to
 * D (truncdim), gauge-fixed with (tol, maxiter).  Writes a new state to *out (release it with
 * imps_state_destroy); its bond dimensions come from imps_state_bonds. */
int imps_mult_guess(const imps_mpo* W, const imps_state* psi, int D, double tol, int maxiter, imps_state** out,
                    imps_gauge_info* info);
/* MultCache(bra, W, ket) (mult.jl:93-197): the :LM fixed points of the <bra|W|ket>
 * transfer matrices (Arnoldi, krylovdim 30, eager, from a deterministic start vector in place
 * of the reference's randn), the other sites by ternary pushes (transfermatrix.jl:77-107),
 * every GR at unit norm and GL[l+1] scaled so that <bra.C[l], mapC(l)> = 1.  bra, W and ket
 * are borrowed and must outlive the object; sweeps change bra in place. */
int imps_mult_envs_create(imps_state* bra, const imps_mpo* W, const imps_state* ket, double tol, int maxiter,
                          imps_mult_envs** out, imps_krylov_info* info);
int imps_mult_envs_destroy(imps_mult_envs* envs);
/* lefts[site] (side 0, (bra bond, w, ket bond)) or rights[site] (side 1, (ket bond, w,
 * bra bond)) to the host. */
int imps_mult_envs_get(const imps_mult_envs* envs, int side, int site, double* host);
/* _local_AC(envs, site) (Dl, d, Dr of the bra, mult.jl:294-297) and _local_C(envs, site)
 * (bond right of site, mult.jl:299-303) to the host; either pointer may be NULL. */
int imps_mult_local_maps(imps_mult_envs* envs, int site, double* ac, double* c);
/* calc_galerkin(envs::MultCache, bra) (mult.jl:586-593). */
int imps_mult_galerkin(imps_mult_envs* envs, double* eps);
/* One compression_sweeps! iteration for VOMPS (arithmetics/envs.jl:60-85): local maps and
 * regauge! for every site, gauge_step! with (gauge_tol, gauge_maxiter), the fixed points
 * re-solved warm with (env_tol, env_maxiter), then *eps = the new Galerkin residual. */
int imps_mult_sweep(imps_mult_envs* envs, double gauge_tol, int gauge_maxiter, double env_tol, int env_maxiter,
                    double* eps);

#ifdef __cplusplus
}
#endif

#endif /* IMPS_B200_H */
